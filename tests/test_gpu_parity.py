"""GPU parity: libcuhc.so through its C ABI against the CPU oracle and the
reference library, bit for bit.

The bar is bit-exactness: merge trees (ids, heights, sizes) and core
distances identical to the oracle, which restates the reference's FP32
arithmetic and its (weight, smaller index, larger index) tie order. Minkowski
uses the reference's fast exp2/log2 powers on the device, which the CPU can
not reproduce, so it is checked against the reference library (bit for bit)
or the oracle within rtol 1e-5.
"""

import pathlib

import numpy as np
import pytest

import cuhc_b200 as C
from _data import assert_well_formed, blobs, grid, normal
from cuhc_b200 import _lib
from cuhc_b200._hdbscan import hdbscan_tree
from golden.inputs import GPU_CASES, make_input
from oracle import oracle as O

pytestmark = pytest.mark.gpu
MODES = ["never", "always", "auto"]
REF_GPU = pathlib.Path(__file__).resolve().parent / "golden" / "reference_gpu.npz"


@pytest.fixture
def pruning():
    def run(mode, fn):
        _lib.set_pruning(mode)
        try:
            return fn()
        finally:
            _lib.set_pruning("auto")
    return run


@pytest.mark.parametrize("n", [2, 3, 127, 128, 129, 255, 257, 1000])
@pytest.mark.parametrize("d", [1, 3, 8, 9, 33])
def test_single_linkage_tile_edges(pruning, n, d):
    X = blobs(n, d, seed=n * 100 + d)
    ref = O.single_linkage(X)
    for mode in MODES:
        np.testing.assert_array_equal(pruning(mode, lambda: C.linkage(X, "single")), ref)


@pytest.mark.parametrize("d", [2, 16, 32, 64, 100])
def test_single_linkage_dims(pruning, d):
    X = normal(3000, d, seed=d)
    ref = O.single_linkage(X)
    for mode in ["never", "always"]:
        np.testing.assert_array_equal(pruning(mode, lambda: C.linkage(X, "single")), ref)


@pytest.mark.parametrize("metric", ["sqeuclidean", "manhattan", "chebyshev", "cosine"])
def test_single_linkage_metrics(pruning, metric):
    X = blobs(2000, 6, seed=41)
    ref = O.single_linkage(X, metric=metric)
    for mode in ["never", "always"]:
        Z = pruning(mode, lambda: C.linkage(X, "single", metric=metric, algorithm="mst"))
        np.testing.assert_array_equal(Z, ref)


def test_minkowski(pruning):
    X = blobs(1500, 5, seed=42)
    ref = O.single_linkage(X, metric="minkowski", p=3.0)
    a = pruning("never", lambda: C.linkage(X, "single", metric="minkowski", p=3.0))
    b = pruning("always", lambda: C.linkage(X, "single", metric="minkowski", p=3.0))
    np.testing.assert_array_equal(a, b)
    np.testing.assert_allclose(a[:, 2], ref[:, 2], rtol=1e-5)
    if O.reference_available():
        np.testing.assert_array_equal(
            a, O.reference_linkage(X, "single", "mst", metric="minkowski", p=3.0))


def test_single_linkage_ties(pruning):
    X = grid(20)
    ref = O.single_linkage(X)
    for mode in MODES:
        Z = pruning(mode, lambda: C.linkage(X, "single"))
        np.testing.assert_array_equal(Z, ref)
        assert np.all(Z[:, 2] == 1.0)


def test_single_linkage_duplicates(pruning):
    X = np.repeat(normal(100, 3, seed=5), 5, axis=0)
    ref = O.single_linkage(X)
    for mode in MODES:
        np.testing.assert_array_equal(pruning(mode, lambda: C.linkage(X, "single")), ref)


@pytest.mark.parametrize("k", [1, 2, 5, 25, 64])
@pytest.mark.parametrize("d", [2, 8])
def test_hdbscan_tree(pruning, k, d):
    X = blobs(3000, d, noise=0.1, seed=k + d)
    Z_ref, core_ref = O.hdbscan_tree(X, k)
    for mode in MODES:
        Z, core = pruning(mode, lambda: hdbscan_tree(X, k))
        np.testing.assert_array_equal(core, core_ref)
        np.testing.assert_array_equal(Z, Z_ref)


@pytest.mark.parametrize("alpha", [0.7, 1.5])
def test_hdbscan_alpha(pruning, alpha):
    X = blobs(2000, 3, noise=0.1, seed=7)
    Z_ref, core_ref = O.hdbscan_tree(X, 10, alpha=alpha)
    for mode in ["never", "always"]:
        Z, core = pruning(mode, lambda: hdbscan_tree(X, 10, alpha=alpha))
        np.testing.assert_array_equal(core, core_ref)
        np.testing.assert_array_equal(Z, Z_ref)


@pytest.mark.parametrize("metric", ["manhattan", "chebyshev", "cosine"])
def test_hdbscan_metrics(metric):
    X = blobs(1500, 4, noise=0.1, seed=8)
    Z_ref, core_ref = O.hdbscan_tree(X, 7, metric=metric)
    Z, core = hdbscan_tree(X, 7, metric=metric)
    np.testing.assert_array_equal(core, core_ref)
    np.testing.assert_array_equal(Z, Z_ref)


def test_hdbscan_duplicates_core_zero():
    X = np.repeat(normal(50, 3, seed=3), 4, axis=0)
    _, core = hdbscan_tree(X, 4)
    assert np.all(core == 0.0)
    _, core = hdbscan_tree(X, 5)
    assert np.all(core > 0.0)


def test_hdbscan_large_k():
    X = blobs(1200, 6, seed=9)
    Z_ref, core_ref = O.hdbscan_tree(X, 200)
    Z, core = hdbscan_tree(X, 200)
    np.testing.assert_array_equal(core, core_ref)
    np.testing.assert_array_equal(Z, Z_ref)


@pytest.mark.parametrize("metric", ["euclidean", "sqeuclidean", "manhattan", "chebyshev",
                                    "cosine"])
@pytest.mark.parametrize("shape", [(1, 1), (7, 3), (129, 9), (300, 64), (257, 100)])
def test_pairwise_distances(metric, shape):
    X = normal(*shape, seed=shape[0])
    np.testing.assert_array_equal(C.pairwise_distances(X, metric=metric),
                                  O.pairwise(X, metric=metric))


def test_pairwise_two_inputs():
    X, Y = normal(150, 20, seed=1), normal(333, 20, seed=2) + 0.5
    np.testing.assert_array_equal(C.pairwise_distances(X, Y), O.pairwise(X, Y))


def test_config1_full_size():
    """20,000 x 32 N(0,1), seed 0: the tree equals the oracle's bit for bit."""
    X = np.random.default_rng(0).standard_normal((20000, 32)).astype(np.float32)
    np.testing.assert_array_equal(C.linkage(X, "single"), O.single_linkage(X))


def test_hdbscan_large_properties(pruning):
    """At 200,000 points: pruned and unpruned trees identical, well formed,
    core distances equal the oracle's on a sample of rows."""
    rng = np.random.default_rng(1)
    centres = rng.uniform(-10, 10, (20, 8))
    X = (np.repeat(centres, 9000, axis=0) + rng.standard_normal((180000, 8)))
    X = np.vstack([X, rng.uniform(X.min(0), X.max(0), (20000, 8))]).astype(np.float32)
    X = X[rng.permutation(len(X))]
    Z1, core1 = pruning("always", lambda: hdbscan_tree(X, 25))
    Z2, core2 = pruning("never", lambda: hdbscan_tree(X, 25))
    np.testing.assert_array_equal(core1, core2)
    np.testing.assert_array_equal(Z1, Z2)
    assert_well_formed(Z1, len(X))
    rows = (0, 300)
    np.testing.assert_array_equal(core1[:300], O.core_distances(X, 25, rows=rows))


@pytest.mark.skipif(not REF_GPU.exists(), reason="reference GPU fixtures not generated")
@pytest.mark.parametrize("name", [k for k, v in GPU_CASES.items() if v["kind"] in
                                  ("single", "hdbscan")])
def test_matches_reference_fixtures(pruning, name):
    ref = np.load(REF_GPU)
    spec = GPU_CASES[name]
    X = make_input(spec)
    for mode in ["never", "always"]:
        if spec["kind"] == "single":
            np.testing.assert_array_equal(pruning(mode, lambda: C.linkage(X, "single")),
                                          ref[f"{name}/Z"])
        else:
            Z, core = pruning(mode, lambda: hdbscan_tree(X, spec["k"]))
            np.testing.assert_array_equal(core, ref[f"{name}/core"])
            np.testing.assert_array_equal(Z, ref[f"{name}/Z"])


@pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref not built")
def test_matches_reference_library_live():
    X = blobs(4000, 8, noise=0.1, seed=77)
    np.testing.assert_array_equal(C.linkage(X, "single"),
                                  O.reference_linkage(X, "single", "mst", pruning="never"))
    Z_ref, core_ref = O.reference_hdbscan_tree(X, 25, pruning="never")
    Z, core = hdbscan_tree(X, 25)
    np.testing.assert_array_equal(core, core_ref)
    np.testing.assert_array_equal(Z, Z_ref)


def test_prune_stats_count_tiles():
    X = blobs(20000, 2, centers=30, seed=30)
    _lib.prune_stats()
    _lib.set_pruning("always")
    try:
        C.linkage(X, "single")
    finally:
        _lib.set_pruning("auto")
    computed, total = _lib.prune_stats()
    assert total > 0 and computed < 0.2 * total


def test_launch_counter_moves():
    before = _lib.launch_count()
    C.linkage(normal(500, 4, seed=1), "single")
    assert _lib.launch_count() > before
