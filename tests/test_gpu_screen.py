"""GPU: the tensor-core screened passes give exactly the plain passes'
results (and the oracle's), across dimensions, tile edges, ties, metrics,
mutual reachability, Ward, pruning modes."""

import numpy as np
import pytest

import cuhc_b200 as C
from _data import blobs, grid, normal
from cuhc_b200 import _lib
from cuhc_b200._hdbscan import hdbscan_tree
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture
def modes():
    def run(screen, prune, fn):
        _lib.set_screen(screen)
        _lib.set_pruning(prune)
        try:
            return fn()
        finally:
            _lib.set_screen("auto")
            _lib.set_pruning("auto")
    return run


@pytest.mark.parametrize("n, d", [(2, 3), (127, 1), (129, 8), (300, 2), (1000, 5), (2000, 16),
                                  (3000, 32), (257, 31)])
def test_single_linkage(modes, n, d):
    X = blobs(n, d, seed=n + d)
    ref = O.single_linkage(X)
    for prune in ("always", "never"):
        np.testing.assert_array_equal(modes("on", prune, lambda: C.linkage(X, "single")), ref)


@pytest.mark.parametrize("metric", ["euclidean", "sqeuclidean"])
def test_metrics(modes, metric):
    X = normal(1500, 12, seed=3)
    ref = O.single_linkage(X, metric=metric)
    np.testing.assert_array_equal(
        modes("on", "always", lambda: C.linkage(X, "single", metric=metric)), ref)


@pytest.mark.parametrize("k", [1, 5, 25, 64, 150])
@pytest.mark.parametrize("d", [2, 8, 30])
def test_hdbscan(modes, k, d):
    X = blobs(2500, d, noise=0.1, seed=k * 3 + d)
    Z_ref, core_ref = O.hdbscan_tree(X, k)
    for prune in ("always", "never"):
        Z, core = modes("on", prune, lambda: hdbscan_tree(X, k))
        np.testing.assert_array_equal(core, core_ref)
        np.testing.assert_array_equal(Z, Z_ref)


def test_hdbscan_alpha(modes):
    X = blobs(2000, 4, noise=0.1, seed=5)
    Z_ref, core_ref = O.hdbscan_tree(X, 10, alpha=0.6)
    Z, core = modes("on", "always", lambda: hdbscan_tree(X, 10, alpha=0.6))
    np.testing.assert_array_equal(core, core_ref)
    np.testing.assert_array_equal(Z, Z_ref)


def test_ties_and_duplicates(modes):
    for X in (grid(24), np.repeat(normal(80, 3, seed=7), 5, axis=0)):
        ref = O.single_linkage(X)
        np.testing.assert_array_equal(modes("on", "always", lambda: C.linkage(X, "single")), ref)
        Z_ref, core_ref = O.hdbscan_tree(X, 6)
        Z, core = modes("on", "always", lambda: hdbscan_tree(X, 6))
        np.testing.assert_array_equal(core, core_ref)
        np.testing.assert_array_equal(Z, Z_ref)


def test_far_from_origin(modes):
    X = (1e4 + blobs(1200, 6, seed=9)).astype(np.float32)
    ref = O.single_linkage(X)
    np.testing.assert_array_equal(modes("on", "always", lambda: C.linkage(X, "single")), ref)


def test_ward_screen_matches_plain(modes):
    X = blobs(3000, 16, seed=52)
    plain = modes("off", "always", lambda: C.linkage(X, "ward"))
    screened = modes("on", "always", lambda: C.linkage(X, "ward"))
    np.testing.assert_array_equal(screened, plain)


def test_large_screen_matches_plain(modes):
    rng = np.random.default_rng(1)
    centres = rng.uniform(-10, 10, (20, 8))
    X = (np.repeat(centres, 9000, axis=0) + rng.standard_normal((180000, 8)))
    X = np.vstack([X, rng.uniform(X.min(0), X.max(0), (20000, 8))]).astype(np.float32)
    X = X[rng.permutation(len(X))]
    Z1, c1 = modes("on", "auto", lambda: hdbscan_tree(X, 25))
    Z2, c2 = modes("off", "auto", lambda: hdbscan_tree(X, 25))
    np.testing.assert_array_equal(c1, c2)
    np.testing.assert_array_equal(Z1, Z2)
    Y = normal(100000, 32, seed=4)
    np.testing.assert_array_equal(modes("on", "auto", lambda: C.linkage(Y, "single")),
                                  modes("off", "auto", lambda: C.linkage(Y, "single")))


def cosine_cases():
    """Cosine data: blobs, the same with every point scaled by a random
    factor in [1e-6, 1e6] (the distance ignores it; squared norms stay inside
    the screen's [2^-60, 2^60]), zero points, exact duplicates and
    antiparallel copies."""
    rng = np.random.default_rng(21)
    X = blobs(1500, 16, noise=0.1, seed=21)
    scaled = (X * np.exp(rng.uniform(np.log(1e-6), np.log(1e6), (len(X), 1)))).astype(np.float32)
    special = X[:400].copy()
    special[:10] = 0.0                      # zero points: distance 1 to everything
    special[10:60] = special[60:110]        # duplicates: distance 0
    special[110:160] = -special[160:210]    # antiparallel: distance 2
    return {"blobs": X, "scaled": scaled, "special": special}


@pytest.mark.parametrize("case", ["blobs", "scaled", "special"])
def test_cosine_screened(modes, case):
    X = cosine_cases()[case]
    ref = O.single_linkage(X, metric="cosine")
    _lib.set_timing(True)
    _lib.kernel_timing()
    try:
        Z = modes("on", "auto", lambda: C.linkage(X, "single", metric="cosine"))
        timing = _lib.kernel_timing()
    finally:
        _lib.set_timing(False)
    np.testing.assert_array_equal(Z, ref)
    assert timing["screen_pass"][1] > 0, timing  # the screened kernel ran
    Z_ref, core_ref = O.hdbscan_tree(X, 7, metric="cosine")
    Z, core = modes("on", "auto", lambda: hdbscan_tree(X, 7, metric="cosine"))
    np.testing.assert_array_equal(core, core_ref)
    np.testing.assert_array_equal(Z, Z_ref)


@pytest.mark.parametrize("d", [3, 8, 31, 32])
def test_cosine_dimensions(modes, d):
    X = normal(1200, d, seed=d)
    ref = O.single_linkage(X, metric="cosine")
    np.testing.assert_array_equal(
        modes("on", "auto", lambda: C.linkage(X, "single", metric="cosine")), ref)


def test_cosine_outside_norm_range_runs_plain(modes):
    """Squared norms below 2^-60 (the reference's norm product could
    underflow there): the screen steps aside and the plain pass gives the
    oracle's tree."""
    X = (normal(600, 6, seed=4) * np.float32(1e-20)).astype(np.float32)
    ref = O.single_linkage(X, metric="cosine")
    _lib.set_timing(True)
    _lib.kernel_timing()
    try:
        Z = modes("on", "auto", lambda: C.linkage(X, "single", metric="cosine"))
        timing = _lib.kernel_timing()
    finally:
        _lib.set_timing(False)
    np.testing.assert_array_equal(Z, ref)
    assert timing["screen_pass"][1] == 0, timing
