"""The CPU oracle, pinned before it is trusted (no GPU needed).

- Single linkage against scipy's trees stored in tests/golden/cpu.npz, at
  the reference's own contract (tests/test_mst.py:18-30 of shangar21/cuhc):
  merges exact, heights to rtol 1e-4 (float32 vs float64);
- core distances against a float64 NumPy sort;
- condensed trees row for row against the reference's cuhc_condense_tree
  (stored outputs; and live when oracle/_ref was built here);
- MST invariants: n - 1 edges, a spanning tree, minimal under the edge order
  (cut property checked exhaustively on small inputs);
- against the reference library's GPU outputs, when the fixture exists.
"""

import pathlib

import numpy as np
import pytest

from _data import assert_well_formed, blobs, grid, normal
from golden.inputs import CPU_CASES, GPU_CASES, make_input
from oracle import oracle as O

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"
CPU = np.load(GOLDEN / "cpu.npz")


@pytest.mark.parametrize("name", [k for k, v in CPU_CASES.items() if v["kind"] == "single"])
def test_single_linkage_matches_scipy(name):
    X = make_input(CPU_CASES[name])
    Z = O.single_linkage(X)
    ref = CPU[f"{name}/Z"]
    np.testing.assert_array_equal(np.sort(Z[:, :2], axis=1), np.sort(ref[:, :2], axis=1))
    np.testing.assert_allclose(Z[:, 2], ref[:, 2], rtol=1e-4, atol=1e-5)
    np.testing.assert_array_equal(Z[:, 3], ref[:, 3])


@pytest.mark.parametrize("k", [1, 2, 7, 25, 40])
def test_core_distances_match_numpy(k):
    X = blobs(300, 5, seed=k)
    D = np.sqrt(((X[:, None, :].astype(np.float64) - X[None]) ** 2).sum(-1))
    np.fill_diagonal(D, 0.0)
    np.testing.assert_allclose(O.core_distances(X, k), np.sort(D, axis=1)[:, k - 1],
                               rtol=1e-5, atol=1e-6)


def test_duplicates_have_zero_core():
    X = np.repeat(normal(50, 3, seed=3), 4, axis=0)
    assert np.all(O.core_distances(X, 4) == 0.0)
    assert np.all(O.core_distances(X, 5) > 0.0)


@pytest.mark.parametrize("name", [k for k, v in CPU_CASES.items() if v["kind"] == "condense"])
def test_condense_matches_reference_fixture(name):
    Z = CPU[f"{name}/tree"]
    for mcs in CPU_CASES[name]["mcs"]:
        ours = O.condense_tree(Z, mcs)
        for field, array in zip(("parent", "child", "lambda", "size"), ours):
            np.testing.assert_array_equal(array, CPU[f"{name}/mcs{mcs}/{field}"])


@pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("mcs", [2, 5, 25, 100])
def test_condense_matches_reference_live(mcs):
    Z, _ = O.hdbscan_tree(blobs(3000, 8, noise=0.1, seed=4), 5)
    for ours, ref in zip(O.condense_tree(Z, mcs), O.reference_condense_tree(Z, mcs)):
        np.testing.assert_array_equal(ours, ref)


def _edge_key(w, u, v):
    return (np.float32(w), min(u, v), max(u, v))


@pytest.mark.parametrize("X", [normal(60, 3, seed=1), grid(8), blobs(80, 2, seed=2)],
                         ids=["normal", "grid", "blobs"])
def test_mst_is_minimal_under_the_edge_order(X):
    """Cut property, exhaustively: every MST edge is the lightest edge, under
    (weight, min, max), across the cut it closes."""
    n = len(X)
    u, v, w = O.mst(X)
    D = O.pairwise(X)
    assert len(u) == n - 1
    parent = list(range(n))

    def find(a):
        while parent[a] != a:
            a = parent[a]
        return a

    order = sorted(range(n - 1), key=lambda i: _edge_key(w[i], u[i], v[i]))
    for i in order:
        ru, rv = find(u[i]), find(v[i])
        assert ru != rv
        # Lightest edge leaving the component of u (Kruskal's order).
        comp = [p for p in range(n) if find(p) == ru]
        best = min(_edge_key(D[a, b], a, b) for a in comp for b in range(n) if find(b) != ru)
        assert best == _edge_key(w[i], u[i], v[i])
        parent[ru] = rv


def test_grid_tree_is_well_formed():
    X = grid(20)
    Z = O.single_linkage(X)
    assert_well_formed(Z, len(X))
    assert np.all(Z[:, 2] == 1.0)


def test_hdbscan_tree_mutual_reachability_bounds():
    X = blobs(800, 4, noise=0.1, seed=9)
    Z, core = O.hdbscan_tree(X, 10)
    assert_well_formed(Z, len(X))
    # Every merge height is at least the smaller core distance involved.
    assert np.all(np.diff(Z[:, 2]) >= 0)
    assert Z[0, 2] >= core.min()


def test_nearest_other_component_ties_to_lower_index():
    # Four points on a line at equal spacing: ties everywhere.
    X = np.array([[0.0], [1.0], [2.0], [3.0]], dtype=np.float32)
    nearest = O.nearest_other_component(X, np.arange(4))
    assert [int(k & 0xFFFFFFFF) for k in nearest] == [1, 0, 1, 2]


REF_GPU = GOLDEN / "reference_gpu.npz"


@pytest.mark.skipif(not REF_GPU.exists(), reason="reference GPU fixtures not generated")
@pytest.mark.parametrize("name", [k for k, v in GPU_CASES.items() if v["kind"] in
                                  ("single", "hdbscan")])
def test_oracle_matches_reference_gpu_outputs(name):
    """The oracle equals the reference library itself, bit for bit."""
    ref = np.load(REF_GPU)
    spec = GPU_CASES[name]
    X = make_input(spec)
    if spec["kind"] == "single":
        np.testing.assert_array_equal(O.single_linkage(X), ref[f"{name}/Z"])
    else:
        Z, core = O.hdbscan_tree(X, spec["k"])
        np.testing.assert_array_equal(core, ref[f"{name}/core"])
        np.testing.assert_array_equal(Z, ref[f"{name}/Z"])
