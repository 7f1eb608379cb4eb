"""scikit-learn compatible AgglomerativeClustering on the exact GPU merge
trees (same parameters, defaults and fitted attributes as
sklearn.cluster.AgglomerativeClustering, plus `algorithm`)."""

import numbers

import numpy as np
from sklearn.base import BaseEstimator, ClusterMixin

from ._distances import as_points
from ._linkage import LINKAGE_IDS, cut_tree, linkage, resolve_algorithm, validate_linkage


class AgglomerativeClustering(ClusterMixin, BaseEstimator):
    """Exact agglomerative clustering on the GPU.

    Parameters: n_clusters (or distance_threshold, exactly one of them),
    metric, linkage ("ward", "complete", "average", "single"),
    compute_distances, algorithm ("auto", "dense", "mst", "rnn", "nn_chain").
    Fitted: labels_, n_clusters_, children_, distances_ (with
    compute_distances or distance_threshold), n_leaves_, n_features_in_,
    n_connected_components_.
    """

    def __init__(self, n_clusters=2, *, metric="euclidean", linkage="ward",
                 distance_threshold=None, compute_distances=False, algorithm="auto"):
        self.n_clusters = n_clusters
        self.metric = metric
        self.linkage = linkage
        self.distance_threshold = distance_threshold
        self.compute_distances = compute_distances
        self.algorithm = algorithm

    def _check_params(self):
        if (self.n_clusters is None) == (self.distance_threshold is None):
            raise ValueError("Exactly one of n_clusters and distance_threshold has to be set, "
                             "and the other needs to be None.")
        if self.n_clusters is not None and (
                not isinstance(self.n_clusters, numbers.Integral) or self.n_clusters < 1):
            raise ValueError(f"n_clusters must be a positive integer, got {self.n_clusters!r}")
        if self.linkage not in LINKAGE_IDS:
            raise ValueError(f"linkage must be one of {list(LINKAGE_IDS)}, got {self.linkage!r}")
        validate_linkage(self.linkage, self.metric)
        resolve_algorithm(self.algorithm, self.linkage)

    def fit(self, X, y=None):
        self._check_params()
        X = as_points(X, "X")
        n = X.shape[0]
        if self.n_clusters is not None and self.n_clusters > n:
            raise ValueError(f"Cannot extract more clusters ({self.n_clusters}) than samples ({n})")
        Z = linkage(X, method=self.linkage, metric=self.metric, algorithm=self.algorithm)
        if self.distance_threshold is not None:
            # Merges at or above the threshold split clusters (sklearn's rule).
            self.n_clusters_ = int(np.count_nonzero(Z[:, 2] >= self.distance_threshold)) + 1
        else:
            self.n_clusters_ = int(self.n_clusters)
        self.labels_ = cut_tree(Z, n - self.n_clusters_)
        self.children_ = Z[:, :2].astype(np.intp)
        if self.compute_distances or self.distance_threshold is not None:
            self.distances_ = Z[:, 2].copy()
        self.n_leaves_ = n
        self.n_features_in_ = X.shape[1]
        self.n_connected_components_ = 1
        return self

    def fit_predict(self, X, y=None):
        return self.fit(X).labels_
