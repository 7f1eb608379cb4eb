"""AgglomerativeClustering on the exact GPU merge trees.

Follows the documented contract of sklearn.cluster.AgglomerativeClustering:
the same constructor parameters and defaults (plus `algorithm`, the tree
builder of `linkage`), the same fitted attributes, and the same flat cut --
with `distance_threshold` set, every merge whose height is at or above the
threshold is undone, so the cut keeps the merges strictly below it.
"""

import numbers

import numpy as np
from sklearn.base import BaseEstimator, ClusterMixin

from ._distances import as_points, device_points
from ._linkage import LINKAGE_IDS, cut_tree, linkage, resolve_algorithm, validate_linkage


class AgglomerativeClustering(ClusterMixin, BaseEstimator):
    """Exact agglomerative clustering on the GPU.

    Parameters: n_clusters (or distance_threshold: set exactly one),
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

    def _flat_cut_size(self, heights, n_samples):
        """Clusters of the flat cut: n_clusters, or the points minus the
        merges strictly below distance_threshold."""
        if self.distance_threshold is None:
            return int(self.n_clusters)
        below = np.asarray(heights) < self.distance_threshold
        return n_samples - int(below.sum())

    def _validate(self, n_samples):
        by_count = self.n_clusters is not None
        by_height = self.distance_threshold is not None
        if by_count == by_height:
            # scikit-learn's own wording: callers match on it.
            raise ValueError("Exactly one of n_clusters and distance_threshold has to be set, "
                             "and the other needs to be None.")
        if self.linkage not in LINKAGE_IDS:
            raise ValueError(f"unknown linkage {self.linkage!r}; expected one of "
                             f"{sorted(LINKAGE_IDS)}")
        validate_linkage(self.linkage, self.metric)
        resolve_algorithm(self.algorithm, self.linkage)
        if by_count:
            valid = isinstance(self.n_clusters, numbers.Integral) and self.n_clusters >= 1
            if not valid:
                raise ValueError(f"n_clusters must be an integer >= 1, got {self.n_clusters!r}")
            if self.n_clusters > n_samples:
                raise ValueError(f"n_clusters={self.n_clusters} exceeds the {n_samples} samples")

    def fit(self, X, y=None):
        device = device_points(X, "X")  # GPU arrays are read in place
        points = X if device is not None else as_points(X, "X")
        n_samples, n_features = device.shape if device is not None else points.shape
        self._validate(n_samples)
        tree = linkage(points, method=self.linkage, metric=self.metric, algorithm=self.algorithm)
        heights = tree[:, 2]
        clusters = self._flat_cut_size(heights, n_samples)
        self.n_leaves_ = n_samples
        self.n_features_in_ = n_features
        self.n_connected_components_ = 1  # every tree here joins all points
        self.children_ = tree[:, :2].astype(np.intp)
        self.n_clusters_ = clusters
        self.labels_ = cut_tree(tree, n_samples - clusters)
        if self.distance_threshold is not None or self.compute_distances:
            self.distances_ = np.array(heights, dtype=np.float64)
        return self

    def fit_predict(self, X, y=None):
        return self.fit(X).labels_
