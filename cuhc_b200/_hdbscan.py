"""HDBSCAN: the GPU single-linkage tree of mutual reachability, condensing,
and cluster extraction with scikit-learn 1.9's semantics."""

import numpy as np

from . import _lib
from ._distances import METRIC_IDS, as_points, check_distance_range

NOISE = -1
# Core-distance methods of the C ABI (reference hdbscan.cuh:324).
CORE_METHOD_IDS = {"auto": 0, "fused": 1, "radix": 2}


def hdbscan_tree(X, min_samples, metric="euclidean", alpha=1.0, p=2.0, core_method="auto"):
    """(Z, core): the (n-1, 4) single-linkage tree of the mutual reachability
    distance max(core_a, core_b, d(a, b) / alpha) and the core distances
    (distance to the min_samples-th nearest point, the point itself first)."""
    X = as_points(X, "X")
    check_distance_range(X, metric, p, scale=1.0 / alpha)
    n = X.shape[0]
    tree = np.empty((max(n - 1, 0), 4), dtype=np.float64)
    core = np.empty(n, dtype=np.float32)
    _lib.check(_lib.lib.cuhc_hdbscan_tree(
        _lib.float_ptr(X), n, X.shape[1], METRIC_IDS[metric], float(p), int(min_samples),
        float(alpha), CORE_METHOD_IDS[core_method], _lib.double_ptr(tree), _lib.float_ptr(core)))
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
