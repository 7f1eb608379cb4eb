"""GPU: Ward (RNN rounds, NN-chain, dense tail), dense complete / average
linkage, the estimators, against the reference library (bit for bit, when
oracle/_ref is built or its fixtures exist) and scikit-learn (its own test
contract: merges exact, heights rtol 1e-4 / atol 1e-5)."""

import pathlib

import numpy as np
import pytest
from scipy.cluster.hierarchy import fcluster as scipy_fcluster

import cuhc_b200 as C
from _data import (assert_same_dendrogram, assert_same_partition, assert_well_formed, blobs,
                   normal, subtree_sizes)
from cuhc_b200 import _lib
from cuhc_b200._linkage import _ward_rnn_with_options
from golden.inputs import GPU_CASES, make_input
from oracle import oracle as O

pytestmark = pytest.mark.gpu
REF_GPU = pathlib.Path(__file__).resolve().parent / "golden" / "reference_gpu.npz"
RTOL, ATOL = 1e-4, 1e-5


def sklearn_tree(X, method, metric="euclidean"):
    from sklearn.cluster import AgglomerativeClustering  # noqa: PLC0415
    from sklearn.metrics import pairwise_distances  # noqa: PLC0415
    X64 = X.astype(np.float64)
    if method == "ward":
        m = AgglomerativeClustering(n_clusters=None, distance_threshold=0.0, linkage="ward")
        m.fit(X64)
    else:
        m = AgglomerativeClustering(n_clusters=None, distance_threshold=0.0, linkage=method,
                                    metric="precomputed")
        m.fit(pairwise_distances(X64, metric=metric))
    n = len(X)
    return np.column_stack([m.children_, m.distances_, subtree_sizes(m.children_, n)])


@pytest.mark.parametrize("n", [2, 3, 127, 128, 129, 600])
@pytest.mark.parametrize("d", [1, 7, 64])
def test_ward_rnn_matches_sklearn(n, d):
    X = blobs(n, d, seed=n + d)
    Z = C.linkage(X, "ward", algorithm="rnn")
    assert_same_dendrogram(Z, sklearn_tree(X, "ward"), RTOL, ATOL)


@pytest.mark.parametrize("name", [k for k, v in GPU_CASES.items() if v["kind"] == "ward"])
def test_ward_rnn_matches_reference_bits(name):
    if not REF_GPU.exists():
        pytest.skip("reference fixtures missing")
    X = make_input(GPU_CASES[name])
    for mode in ["never", "always"]:
        _lib.set_pruning(mode)
        try:
            Z = C.linkage(X, "ward", algorithm="rnn")
        finally:
            _lib.set_pruning("auto")
        np.testing.assert_array_equal(Z, np.load(REF_GPU)[f"{name}/Z"])


def test_ward_rnn_deterministic():
    X = blobs(4000, 4, seed=55)
    first = C.linkage(X, "ward")
    for _ in range(3):
        np.testing.assert_array_equal(C.linkage(X, "ward"), first)


@pytest.mark.parametrize("tail", ["dense", "chain"])
def test_ward_tails(tail):
    X = blobs(1500, 8, seed=53)
    ref = sklearn_tree(X, "ward")
    Z = _ward_rnn_with_options(X, min_progress=1.0, allow_dense=(tail == "dense"))
    assert_same_dendrogram(Z, ref, RTOL, ATOL)
    if tail == "dense":
        assert_same_dendrogram(_ward_rnn_with_options(X, 0.0, dense_below=len(X)), ref, RTOL, ATOL)
        assert_same_dendrogram(_ward_rnn_with_options(X, 0.0, dense_below=300), ref, RTOL, ATOL)


def test_ward_worst_case_hands_over():
    x = 1.01 ** np.arange(1200, dtype=np.float64)
    X = ((x - x[0]) / (x[-1] - x[0]))[:, None].astype(np.float32)
    ref = sklearn_tree(X, "ward")
    for allow_dense in (True, False):
        assert_same_dendrogram(_ward_rnn_with_options(X, 0.01, allow_dense=allow_dense), ref,
                               RTOL, ATOL)


@pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("options", [(1.0, 0, 1), (1.0, 0, 0), (0.0, 400, 1)])
def test_ward_tails_match_reference_bits(options):
    X = blobs(1500, 6, seed=54)
    ref = O.reference()
    Z_ref = np.empty((len(X) - 1, 4))
    import ctypes  # noqa: PLC0415
    f32, f64 = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double)
    O.reference_check(ref.cuhc_set_pruning(2))
    O.reference_check(ref.cuhc_ward_rnn_with_options(
        X.ctypes.data_as(f32), len(X), X.shape[1], options[0], options[1], options[2],
        Z_ref.ctypes.data_as(f64)))
    Z = _ward_rnn_with_options(X, options[0], dense_below=options[1], allow_dense=bool(options[2]))
    np.testing.assert_array_equal(Z, Z_ref)


@pytest.mark.parametrize("n", [2, 3, 255, 256, 257, 600])
def test_nn_chain_matches_sklearn(n):
    X = blobs(n, 7, seed=n)
    assert_same_dendrogram(C.linkage(X, "ward", algorithm="nn_chain"), sklearn_tree(X, "ward"),
                           RTOL, ATOL)


@pytest.mark.skipif(not O.reference_available(), reason="oracle/_ref not built")
def test_nn_chain_and_dense_match_reference_bits():
    X = blobs(2000, 10, seed=41)
    for algorithm in ("nn_chain", "dense"):
        Z_ref = O.reference_linkage(X, "ward", algorithm)
        np.testing.assert_array_equal(C.linkage(X, "ward", algorithm=algorithm), Z_ref)
    for method in ("complete", "average", "single"):
        for metric in ("euclidean", "manhattan", "cosine"):
            Z_ref = O.reference_linkage(X[:700], method, "dense", metric=metric)
            np.testing.assert_array_equal(
                C.linkage(X[:700], method, metric=metric, algorithm="dense"), Z_ref)


@pytest.mark.parametrize("method", ["single", "complete", "average", "ward"])
@pytest.mark.parametrize("n", [2, 3, 130, 400])
def test_dense_matches_sklearn(method, n):
    X = blobs(n, 8, seed=n)
    Z = C.linkage(X, method, algorithm="dense")
    ref = sklearn_tree(X, method)
    np.testing.assert_array_equal(np.sort(Z[:, :2], axis=1), np.sort(ref[:, :2], axis=1))
    np.testing.assert_allclose(Z[:, 2], ref[:, 2], rtol=RTOL, atol=ATOL)


@pytest.mark.parametrize("method", ["single", "complete", "average", "ward"])
def test_duplicates_give_valid_trees(method):
    X = np.repeat(normal(40, 3, seed=9), 5, axis=0)
    Z = C.linkage(X, method)
    assert_well_formed(Z, len(X))
    np.testing.assert_allclose(Z[:160, 2], 0.0, atol=ATOL)


def test_estimators():
    X = blobs(600, 5, seed=15)
    for linkage in ("single", "complete", "average", "ward"):
        ours = C.AgglomerativeClustering(n_clusters=6, linkage=linkage).fit(X)
        from sklearn.cluster import AgglomerativeClustering  # noqa: PLC0415
        ref = AgglomerativeClustering(n_clusters=6, linkage=linkage).fit(X.astype(np.float64))
        assert_same_partition(ours.labels_, ref.labels_)
    model = C.HDBSCAN(min_cluster_size=10).fit(blobs(800, 3, noise=0.1, seed=3))
    assert model.labels_.shape == (800,) and model.probabilities_.shape == (800,)


def test_hdbscan_estimator_matches_sklearn_extraction():
    from sklearn.cluster._hdbscan._linkage import HIERARCHY_dtype  # noqa: PLC0415
    from sklearn.cluster._hdbscan._tree import tree_to_labels  # noqa: PLC0415
    X = blobs(1500, 4, centers=6, noise=0.1, seed=21)
    ours = C.HDBSCAN(min_cluster_size=15).fit(X)
    Z = ours._single_linkage_tree_
    tree = np.empty(len(Z), dtype=HIERARCHY_dtype)
    tree["left_node"], tree["right_node"], tree["value"], tree["cluster_size"] = \
        Z[:, 0], Z[:, 1], Z[:, 2], Z[:, 3]
    labels, probs = tree_to_labels(tree, min_cluster_size=15)
    np.testing.assert_array_equal(ours.labels_, labels)
    np.testing.assert_array_equal(ours.probabilities_, probs)


def test_hdbscan_no_ties_matches_sklearn_end_to_end():
    from sklearn.cluster import HDBSCAN as SkHDBSCAN  # noqa: PLC0415
    X = blobs(600, 4, centers=6, noise=0.1, seed=20)
    ours = C.HDBSCAN(min_cluster_size=20, min_samples=1).fit(X)
    ref = SkHDBSCAN(min_cluster_size=20, min_samples=1, copy=True).fit(X.astype(np.float64))
    assert_same_partition(ours.labels_, ref.labels_)


def test_fcluster_on_gpu_tree():
    X = blobs(200, 4, seed=5)
    assert len(np.unique(C.fcluster(C.linkage(X, "ward"), 5))) == 5
    Z = C.linkage(X, "average")
    for k in (2, 10, 50):
        assert_same_partition(C.fcluster(Z, k), scipy_fcluster(Z, k, "maxclust"))
