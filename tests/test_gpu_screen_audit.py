"""GPU: the tensor-core screen's bound, checked pair by pair on adversarial
data.

The screened passes rest on one guarantee: for every evaluated pair the
tensor-core value D' is at most the reference's FP32 squared distance s
(plus 2^-70 for flushed subnormal products), so no pair that can win is ever
screened out. With the audit switched on the library checks every evaluated
pair of every screened tile against s and an FP64 recomputation. Each test
below asserts, on data built to stress one term of the error bound, that
  - the audit saw pairs and no violation (D' > s + 2^-70),
  - the smallest slack (s - D') / (e (|x|^2 + |y|^2)) stays positive,
  - the trees (and core distances) equal the CPU oracle's bit for bit.
The FP32 chain the bound must contain is the reference's per-feature
fmaf((a - b), (a - b), acc) (src/distances.cuh:21-33).
"""

import numpy as np
import pytest

import cuhc_b200 as C
from _data import blobs
from cuhc_b200 import _lib
from cuhc_b200._hdbscan import hdbscan_tree
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture
def audited():
    _lib.set_screen("on")
    _lib.set_pruning("always")
    _lib.set_screen_audit(True)
    _lib.screen_audit()
    try:
        yield
    finally:
        _lib.set_screen_audit(False)
        _lib.set_screen("auto")
        _lib.set_pruning("auto")


def assert_bound_held(min_pairs=1, relative=True):
    """No violation; with `relative`, the relative margin was exercised and
    the smallest slack is positive (at underflow scales only the absolute
    2^-70 term applies and no pair takes part in the slack)."""
    audit = _lib.screen_audit()
    assert audit["pairs"] >= min_pairs, audit
    assert audit["violations"] == 0, audit
    if relative:
        assert audit["min_slack"] > 0.0, audit
    else:
        assert not audit["min_slack"] <= 0.0, audit  # NaN: no pair in the relative regime
    return audit


def check_trees(X, k=5):
    np.testing.assert_array_equal(C.linkage(X, "single"), O.single_linkage(X))
    Z, core = hdbscan_tree(X, k)
    Z_ref, core_ref = O.hdbscan_tree(X, k)
    np.testing.assert_array_equal(core, core_ref)
    np.testing.assert_array_equal(Z, Z_ref)


def tight_pairs_in_a_wide_box(n, d, spread, gap, seed):
    """Pairs of points `gap` apart scattered over [-spread, spread]^d: few
    points per unit volume, so tile boxes are wide and the centred norms
    dwarf the distances that decide the tree."""
    rng = np.random.default_rng(seed)
    base = rng.uniform(-spread, spread, (n // 2, d))
    partner = base + gap * rng.standard_normal((n // 2, d))
    return np.ascontiguousarray(np.vstack([base, partner]).astype(np.float32)[rng.permutation(n)])


@pytest.mark.parametrize("d", [7, 8, 9, 31, 32])
def test_feature_counts_at_chunk_edges(audited, d):
    X = blobs(2500, d, centers=6, noise=0.1, seed=40 + d)
    check_trees(X, k=10)
    assert_bound_held()


@pytest.mark.parametrize("d, spread, gap", [(8, 1e3, 1e-3), (16, 1e2, 1e-4), (3, 1e4, 1e-2)])
def test_large_norms_far_from_the_tile_centre(audited, d, spread, gap):
    X = tight_pairs_in_a_wide_box(2000, d, spread, gap, seed=d)
    check_trees(X, k=3)
    assert_bound_held()


def test_offset_far_from_the_origin(audited):
    X = (np.float32(3e5) + blobs(1500, 8, centers=4, seed=3)).astype(np.float32)
    check_trees(X, k=7)
    assert_bound_held()


def test_duplicates_and_near_ties_at_the_row_threshold(audited):
    """Rings of points at one radius from each centre, radii nudged by one
    ulp, and duplicated points: k-th neighbour distances and Borůvka edge
    weights tie or nearly tie at the rows' thresholds."""
    rng = np.random.default_rng(21)
    d, k = 6, 8
    centres = rng.uniform(-20, 20, (60, d)).astype(np.float32)
    pts = [centres]
    for c in centres:
        u = rng.standard_normal((k + 4, d))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        r = np.float32(0.75)
        radii = np.array([r, np.nextafter(r, np.float32(1)), np.nextafter(r, np.float32(0))],
                         np.float32)[rng.integers(0, 3, k + 4)]
        pts.append((c + u * radii[:, None]).astype(np.float32))
    X = np.vstack(pts + [centres[:20]]).astype(np.float32)  # 20 exact duplicates
    X = np.ascontiguousarray(X[rng.permutation(len(X))])
    check_trees(X, k=k)
    assert_bound_held()


def test_integer_grid_exact_ties(audited):
    g = np.stack(np.meshgrid(*[np.arange(9)] * 3), axis=-1).reshape(-1, 3).astype(np.float32)
    check_trees(g, k=6)
    assert_bound_held()


@pytest.mark.parametrize("scale", [2.0 ** -120, 2.0 ** -66, 2.0 ** -30, 2.0 ** 30])
def test_tiny_and_huge_scales(audited, scale):
    """2^-120: every squared difference underflows to 0 in FP32; 2^-66: the
    squared distances are subnormal, far below the absolute 2^-70 term;
    2^-30 and 2^30: ordinary relative rounding at extreme exponents."""
    X = (blobs(1200, 8, centers=5, noise=0.05, seed=8) * np.float32(scale)).astype(np.float32)
    check_trees(X, k=5)
    assert_bound_held(relative=scale > 2.0 ** -60)


def test_ward_rounds(audited):
    X = blobs(3000, 16, centers=8, seed=52)
    screened = C.linkage(X, "ward")
    audit = assert_bound_held()
    _lib.set_screen("off")
    np.testing.assert_array_equal(C.linkage(X, "ward"), screened)
    assert audit["pairs"] > 0


def test_audit_reports_fp64_errors(audited):
    """The FP64 figures are consistent: the reference chain's relative error
    is a few FP32 ulps times d, the screened bound sits below the FP64 value
    by at most a small multiple of the margin times the norms."""
    X = blobs(4000, 8, centers=10, noise=0.1, seed=77)
    hdbscan_tree(X, 25)
    audit = assert_bound_held(min_pairs=10_000)
    assert 0.0 <= audit["max_exact_rel"] < 16 * 2.0 ** -24 * 8, audit
    assert audit["max_bound_gap_rel_norms"] < 0.05, audit
    assert audit["min_slack"] > 0.25, audit


@pytest.mark.parametrize("d", [3, 16, 32])
def test_cosine_bound(audited, d):
    """Cosine: the screened value bounds the reference's FP32 distance
    1 - a.b / sqrt(|a|^2 |b|^2) (src/distances.cuh:69-83) for every pair, on
    points scaled over twelve orders of magnitude, with zero points,
    duplicates and antiparallel pairs (distances 1, 0 and 2)."""
    rng = np.random.default_rng(d)
    X = blobs(1200, d, noise=0.1, seed=d)
    X = (X * np.exp(rng.uniform(np.log(1e-6), np.log(1e6), (len(X), 1)))).astype(np.float32)
    X[:5] = 0.0
    X[5:40] = X[40:75]
    X[75:110] = -X[110:145]
    Z = C.linkage(X, "single", metric="cosine")
    Zh, core = hdbscan_tree(X, 5, metric="cosine")
    assert_bound_held(min_pairs=len(X))
    np.testing.assert_array_equal(Z, O.single_linkage(X, metric="cosine"))
    Z_ref, core_ref = O.hdbscan_tree(X, 5, metric="cosine")
    np.testing.assert_array_equal(core, core_ref)
    np.testing.assert_array_equal(Zh, Z_ref)
