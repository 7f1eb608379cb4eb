"""HDBSCAN: the GPU single-linkage tree of mutual reachability, condensing,
and cluster extraction with scikit-learn 1.9's semantics."""

import numbers

import numpy as np

from . import _lib
from ._distances import (METRIC_IDS, as_points, check_distance_range, device_points,
                         validate_metric)

NOISE = -1
# Core-distance methods of the C ABI (reference hdbscan.cuh:324).
CORE_METHOD_IDS = {"auto": 0, "fused": 1, "radix": 2}


def hdbscan_tree(X, min_samples, metric="euclidean", alpha=1.0, p=2.0, core_method="auto"):
    """(Z, core): the (n-1, 4) single-linkage tree of the mutual reachability
    distance max(core_a, core_b, d(a, b) / alpha) and the core distances
    (distance to the min_samples-th nearest point, the point itself first)."""
    X_dev = device_points(X, "X")
    if X_dev is None:
        X = as_points(X, "X")
        check_distance_range(X, metric, p, scale=1.0 / alpha)
    n, d = X.shape if X_dev is None else X_dev.shape
    tree = np.empty((max(n - 1, 0), 4), dtype=np.float64)
    core = np.empty(n, dtype=np.float32)
    args = (n, d, METRIC_IDS[metric], float(p), int(min_samples), float(alpha),
            CORE_METHOD_IDS[core_method], _lib.double_ptr(tree), _lib.float_ptr(core))
    if X_dev is not None:
        # Points already in GPU memory (CuPy, PyTorch, DLPack): read in place.
        _lib.check(_lib.lib.cuhc_hdbscan_tree_device(X_dev.pointer, *args))
    else:
        _lib.check(_lib.lib.cuhc_hdbscan_tree(_lib.float_ptr(X), *args))
    return tree, core


def condense_tree(Z, min_cluster_size):
    """(parent, child, lambda, child_size) rows of the condensed tree."""
    Z = np.ascontiguousarray(Z, dtype=np.float64)
    n = len(Z) + 1
    capacity = n + 2 * (n // max(int(min_cluster_size), 1)) + 2
    parent, child = np.empty(capacity, np.int64), np.empty(capacity, np.int64)
    lam, size = np.empty(capacity, np.float64), np.empty(capacity, np.int64)
    rows = _lib.lib.cuhc_condense_tree(_lib.double_ptr(Z), n, int(min_cluster_size), capacity,
                                       _lib.int64_ptr(parent), _lib.int64_ptr(child),
                                       _lib.double_ptr(lam), _lib.int64_ptr(size))
    if rows < 0:
        raise RuntimeError(f"condensed tree needs {-rows} rows, {capacity} allocated")
    return (parent[:rows].astype(np.intp), child[:rows].astype(np.intp), lam[:rows],
            size[:rows].astype(np.intp))


# ---------------------------------------------------------------------------
# Extraction (C++, scikit-learn 1.9 semantics) and the estimator

_METHODS = {"eom": 0, "leaf": 1}


def tree_to_labels(Z, min_cluster_size, cluster_selection_method="eom",
                   allow_single_cluster=False, cluster_selection_epsilon=0.0,
                   max_cluster_size=None):
    """(labels, probabilities) of HDBSCAN's flat clustering of the tree Z,
    identical to sklearn's tree_to_labels on the same tree."""
    Z = np.ascontiguousarray(Z, dtype=np.float64)
    n = len(Z) + 1
    labels = np.empty(n, dtype=np.int64)
    probabilities = np.empty(n, dtype=np.float64)
    _lib.check(_lib.lib.cuhc_hdbscan_labels(
        _lib.double_ptr(Z), n, int(min_cluster_size), _METHODS[cluster_selection_method],
        int(bool(allow_single_cluster)), float(cluster_selection_epsilon),
        int(max_cluster_size) if max_cluster_size is not None else 0,
        _lib.int64_ptr(labels), _lib.double_ptr(probabilities)))
    return labels.astype(np.intp), probabilities


try:
    from sklearn.base import BaseEstimator, ClusterMixin
except ImportError:  # pragma: no cover
    BaseEstimator, ClusterMixin = object, object


class HDBSCAN(ClusterMixin, BaseEstimator):
    """Density-based clustering, a drop-in for sklearn.cluster.HDBSCAN with
    the same parameters, defaults and results (labels_, probabilities_),
    plus core_distances_. The n x n distance matrix is never stored.

    Parameters: min_cluster_size (>= 2), min_samples (None: min_cluster_size;
    counts the point itself), cluster_selection_epsilon, max_cluster_size,
    metric (a name in METRIC_IDS; minkowski uses p = 2), alpha (mutual
    reachability max(core_a, core_b, d / alpha)), cluster_selection_method
    ("eom" or "leaf"), allow_single_cluster.
    """

    def __init__(self, min_cluster_size=5, min_samples=None, cluster_selection_epsilon=0.0,
                 max_cluster_size=None, metric="euclidean", alpha=1.0,
                 cluster_selection_method="eom", allow_single_cluster=False):
        self.min_cluster_size = min_cluster_size
        self.min_samples = min_samples
        self.cluster_selection_epsilon = cluster_selection_epsilon
        self.max_cluster_size = max_cluster_size
        self.metric = metric
        self.alpha = alpha
        self.cluster_selection_method = cluster_selection_method
        self.allow_single_cluster = allow_single_cluster

    def _check_params(self):
        def integer(value, low):
            return isinstance(value, numbers.Integral) and value >= low

        if not integer(self.min_cluster_size, 2):
            raise ValueError(f"min_cluster_size must be an integer >= 2, got "
                             f"{self.min_cluster_size!r}")
        if self.min_samples is not None and not integer(self.min_samples, 1):
            raise ValueError(f"min_samples must be None or an integer >= 1, got "
                             f"{self.min_samples!r}")
        if self.max_cluster_size is not None and not integer(self.max_cluster_size, 1):
            raise ValueError(f"max_cluster_size must be None or an integer >= 1, got "
                             f"{self.max_cluster_size!r}")
        if not self.cluster_selection_epsilon >= 0:
            raise ValueError(f"cluster_selection_epsilon must be >= 0, got "
                             f"{self.cluster_selection_epsilon!r}")
        if not self.alpha > 0:
            raise ValueError(f"alpha must be > 0, got {self.alpha!r}")
        if self.cluster_selection_method not in _METHODS:
            raise ValueError(f"cluster_selection_method must be 'eom' or 'leaf', got "
                             f"{self.cluster_selection_method!r}")
        validate_metric(self.metric, 2.0)

    def fit(self, X, y=None):
        self._check_params()
        X_dev = device_points(X, "X")
        if X_dev is None:
            X = as_points(X, "X")
        n, d = X.shape if X_dev is None else X_dev.shape
        k = self.min_cluster_size if self.min_samples is None else self.min_samples
        if k > n:
            raise ValueError(f"min_samples ({k}) must be at most the number of samples ({n})")
        Z, core = hdbscan_tree(X, k, metric=self.metric, alpha=self.alpha)
        self.labels_, self.probabilities_ = tree_to_labels(
            Z, self.min_cluster_size, self.cluster_selection_method, self.allow_single_cluster,
            self.cluster_selection_epsilon, self.max_cluster_size)
        self._single_linkage_tree_ = Z
        self.core_distances_ = core
        self.n_features_in_ = d
        return self

    def fit_predict(self, X, y=None):
        return self.fit(X).labels_
