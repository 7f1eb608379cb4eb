"""Python API validation (no GPU: every case fails before the C call), with
the reference's messages and rules (python/cuhc/_distances.py,
_linkage.py, _estimators.py, _hdbscan.py)."""

import numpy as np
import pytest
from sklearn.base import ClusterMixin, clone

import cuhc_b200 as C
from _data import blobs


def huge_spread(n=200):
    return (1.01 ** np.arange(n, dtype=np.float64) * 1e20)[:, None].astype(np.float32)


@pytest.mark.parametrize("call, message", [
    (lambda: C.pairwise_distances(np.zeros((3, 2)), metric="nope"), "unknown metric"),
    (lambda: C.pairwise_distances(np.zeros((3, 2)), np.zeros((3, 4))), "same number of features"),
    (lambda: C.pairwise_distances(np.zeros(3)), "must be 2D"),
    (lambda: C.pairwise_distances(np.zeros((0, 3))), "non-empty"),
    (lambda: C.pairwise_distances(np.zeros((3, 2)), metric="minkowski", p=0), "positive"),
    (lambda: C.pairwise_distances(np.array([[0.0, np.nan]])), "NaN or infinity"),
    (lambda: C.pairwise_distances(np.zeros((2, 2)), np.array([[np.inf, 0.0]])), "NaN or infinity"),
    (lambda: C.pairwise_distances(huge_spread()), "too large for float32"),
    (lambda: C.linkage(huge_spread(), "single"), "too large for float32"),
    (lambda: C.linkage(huge_spread(), "ward"), "too large for float32"),
    (lambda: C.HDBSCAN().fit(huge_spread()), "too large for float32"),
    (lambda: C.linkage(np.array([[0.0], [1e18]] * 500, dtype=np.float32), "ward"),
     "too large for float32"),
    (lambda: C.linkage(blobs(20), "median-of-means"), "method"),
    (lambda: C.linkage(blobs(20), "ward", metric="manhattan"), "euclidean"),
    (lambda: C.linkage(blobs(20), "complete", algorithm="mst"), "supports linkage"),
    (lambda: C.linkage(blobs(20), "single", algorithm="fastest"), "unknown algorithm"),
    (lambda: C.linkage(blobs(20), "single", algorithm="rnn"), "supports linkage"),
    (lambda: C.linkage(np.where(blobs(50) > 0, blobs(50), np.nan), "single"), "NaN"),
    (lambda: C.AgglomerativeClustering(linkage="ward", algorithm="mst").fit(blobs(20)),
     "supports linkage"),
    (lambda: C.AgglomerativeClustering(n_clusters=None).fit(blobs(20)), "Exactly one"),
    (lambda: C.AgglomerativeClustering(n_clusters=0).fit(blobs(20)), "integer >= 1"),
    (lambda: C.AgglomerativeClustering(n_clusters=30).fit(blobs(20)), "exceeds the 20 samples"),
    (lambda: C.fcluster(np.zeros((3, 4)), 0), "t >= 1"),
    (lambda: C.fcluster(np.zeros((3, 4)), 3, criterion="inconsistent"), "criterion"),
])
def test_rejects_bad_input(call, message):
    with pytest.raises(ValueError, match=message):
        call()


@pytest.mark.parametrize("params, message", [
    ({"min_cluster_size": 1}, "min_cluster_size"),
    ({"min_samples": 0}, "min_samples"),
    ({"min_samples": 1000}, "at most the number of samples"),
    ({"alpha": 0.0}, "alpha"),
    ({"cluster_selection_epsilon": -1.0}, "epsilon"),
    ({"cluster_selection_method": "biggest"}, "cluster_selection_method"),
    ({"metric": "hamming"}, "unknown metric"),
])
def test_hdbscan_rejects_bad_parameters(params, message):
    with pytest.raises(ValueError, match=message):
        C.HDBSCAN(**params).fit(blobs(100))


def test_single_point_linkage_is_empty():
    assert C.linkage(np.zeros((1, 3), np.float32), "single").shape == (0, 4)


def test_estimators_are_sklearn_estimators():
    from sklearn.cluster import HDBSCAN as SkHDBSCAN  # noqa: PLC0415
    model = C.HDBSCAN(min_cluster_size=7, metric="manhattan")
    assert isinstance(model, ClusterMixin)
    assert clone(model).get_params() == model.get_params()
    ours, ref = C.HDBSCAN(), SkHDBSCAN()
    for name in ["min_cluster_size", "min_samples", "cluster_selection_epsilon",
                 "max_cluster_size", "metric", "alpha", "cluster_selection_method",
                 "allow_single_cluster"]:
        assert getattr(ours, name) == getattr(ref, name), name
    agg = C.AgglomerativeClustering(n_clusters=3, linkage="average")
    assert clone(agg).get_params() == agg.get_params()


def test_cut_tree_and_fcluster_match_scipy():
    from scipy.cluster.hierarchy import fcluster, linkage  # noqa: PLC0415
    from _data import assert_same_partition  # noqa: PLC0415
    Z = linkage(blobs(300, seed=4).astype(np.float64), "average")
    for t in (1, 2, 7, 50, 300):
        assert_same_partition(C.fcluster(Z, t), fcluster(Z, t, "maxclust"))
    for q in (0.0, 0.5, 0.9, 1.0):
        t = float(np.quantile(Z[:, 2], q))
        assert_same_partition(C.fcluster(Z, t, "distance"), fcluster(Z, t, "distance"))


def test_metric_table_is_the_reference_table():
    assert C.METRIC_IDS == {"euclidean": 0, "l2": 0, "sqeuclidean": 1, "manhattan": 2,
                            "cityblock": 2, "l1": 2, "chebyshev": 3, "minkowski": 4, "cosine": 5}
    assert C.LINKAGE_IDS == {"single": 0, "complete": 1, "average": 2, "ward": 3}
