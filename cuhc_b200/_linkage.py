"""Merge trees in scipy's linkage format, and flat cuts of them.

Mirrors the reference's python/cuhc/_linkage.py: the same id tables
(LINKAGE_IDS :9, ALGORITHM_IDS :15), the same "auto" choice (:29-46: single
-> mst, ward -> rnn, others -> dense), validation messages, and the same
fcluster / cut_tree semantics (:152-216).
"""

import numpy as np

from . import _lib
from ._distances import (METRIC_IDS, as_points, check_distance_range, device_points,
                         validate_metric)

LINKAGE_IDS = {"single": 0, "complete": 1, "average": 2, "ward": 3}
ALGORITHM_IDS = {"dense": 0, "mst": 1, "nn_chain": 2, "rnn": 3}
# Which linkages each algorithm builds.
_SUPPORTED = {"dense": set(LINKAGE_IDS), "mst": {"single"}, "nn_chain": {"ward"},
              "rnn": {"ward"}}
_AUTO = {"single": "mst", "ward": "rnn"}


def validate_linkage(method, metric):
    if method not in LINKAGE_IDS:
        raise ValueError(f"unknown linkage method {method!r}; choose from {list(LINKAGE_IDS)}")
    if method == "ward" and METRIC_IDS.get(metric) != METRIC_IDS["euclidean"]:
        raise ValueError(f"ward linkage requires metric='euclidean', got {metric!r}")


def resolve_algorithm(algorithm, method):
    """The algorithm that builds `method`; "auto" is the fastest exact one."""
    if algorithm == "auto":
        return _AUTO.get(method, "dense")
    if algorithm not in ALGORITHM_IDS:
        raise ValueError(f"unknown algorithm {algorithm!r}; choose 'auto' or one of "
                         f"{list(ALGORITHM_IDS)}")
    if method not in _SUPPORTED[algorithm]:
        raise ValueError(f"algorithm={algorithm!r} supports linkage "
                         f"{sorted(_SUPPORTED[algorithm])}, not {method!r}")
    return algorithm


def linkage(X, method="single", metric="euclidean", p=2.0, *, algorithm="auto"):
    """Full merge tree of the rows of X, like scipy.cluster.hierarchy.linkage.

    Returns Z, an (n-1, 4) float64 array: row i merges clusters Z[i, 0] and
    Z[i, 1] (points are 0..n-1, row i creates cluster n+i) at height Z[i, 2]
    into a cluster of Z[i, 3] points, rows in order of height. Exact for every
    algorithm: "mst" (single, Borůvka), "rnn" and "nn_chain" (ward), "dense"
    (any linkage, n x n matrix on the GPU).
    """
    validate_linkage(method, metric)
    resolve_algorithm(algorithm, method)
    validate_metric(metric, p)
    algorithm = resolve_algorithm(algorithm, method)
    X_dev = device_points(X, "X")
    if X_dev is not None:
        # Points already in GPU memory (CuPy, PyTorch, DLPack): read in place.
        n, d = X_dev.shape
        tree = np.empty((max(n - 1, 0), 4), dtype=np.float64)
        if n == 1:
            return tree
        status = _lib.lib.cuhc_linkage_device(X_dev.pointer, n, d, METRIC_IDS[metric], float(p),
                                              LINKAGE_IDS[method], ALGORITHM_IDS[algorithm],
                                              _lib.double_ptr(tree))
    else:
        X = as_points(X, "X")
        n, d = X.shape
        # Ward heights grow with cluster size: 2 n_a n_b / (n_a + n_b) <= n.
        check_distance_range(X, metric, p, scale=n if method == "ward" else 1.0)
        tree = np.empty((max(n - 1, 0), 4), dtype=np.float64)
        if n == 1:
            return tree
        status = _lib.lib.cuhc_linkage(_lib.float_ptr(X), n, d, METRIC_IDS[metric], float(p),
                                       LINKAGE_IDS[method], ALGORITHM_IDS[algorithm],
                                       _lib.double_ptr(tree))
    if status == _lib.CUDA_ERROR_OUT_OF_MEMORY and algorithm == "dense":
        hint = " (ward linkage can use algorithm='rnn' instead)" if method == "ward" else ""
        raise MemoryError(f"the dense {n} x {n} distance matrix needs {4 * n * n / 1e9:.1f} GB "
                          f"of GPU memory{hint}")
    _lib.check(status)
    return tree


def _ward_rnn_with_options(X, min_progress, dense_below=0, allow_dense=True):
    """Test hook: Ward by RNN rounds with explicit hand-over settings."""
    X = as_points(X, "X")
    n = X.shape[0]
    tree = np.empty((max(n - 1, 0), 4), dtype=np.float64)
    _lib.check(_lib.lib.cuhc_ward_rnn_with_options(
        _lib.float_ptr(X), n, X.shape[1], float(min_progress), int(dense_below),
        int(bool(allow_dense)), _lib.double_ptr(tree)))
    return tree


def cut_tree(Z, num_merges):
    """Labels 0..k-1 of the leaves after the first num_merges merges of Z."""
    Z = np.asarray(Z)
    n = Z.shape[0] + 1
    up = np.arange(2 * n - 1)
    merged = Z[:num_merges, :2].astype(np.intp)
    created = n + np.arange(num_merges)
    up[merged[:, 0]] = created
    up[merged[:, 1]] = created
    # Pointer doubling: each pass jumps twice as far towards the roots.
    while True:
        nxt = up[up]
        if np.array_equal(nxt, up):
            break
        up = nxt
    return np.unique(up[:n], return_inverse=True)[1]


def fcluster(Z, t, criterion="maxclust"):
    """Flat clusters of a merge tree, like scipy.cluster.hierarchy.fcluster
    for "maxclust" (at most t clusters) and "distance" (merges at height <= t).
    Labels start at 1."""
    Z = np.asarray(Z)
    n = Z.shape[0] + 1
    if criterion == "maxclust":
        if t < 1:
            raise ValueError(f"maxclust needs t >= 1, got {t}")
        num_merges = n - min(int(t), n)
    elif criterion == "distance":
        num_merges = int(np.count_nonzero(Z[:, 2] <= t))
    else:
        raise ValueError(f"unknown criterion {criterion!r}; use 'maxclust' or 'distance'")
    return cut_tree(Z, num_merges) + 1
