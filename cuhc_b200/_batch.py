"""Many small clustering problems in one batched solve per feature count.

Each instance is a (n_i, d) point set with its own min_samples: 0 gives the
single-linkage tree (scipy's linkage format), k >= 1 HDBSCAN's tree of the
mutual reachability distance with min_samples = k (alpha 1). Every tree is
bit-identical to the one the per-instance calls (`linkage(X, "single")`,
`hdbscan_tree(X, k)`) return; the batch only removes their per-call launch,
allocation and synchronisation costs. No counterpart in the reference.
"""

import ctypes

import numpy as np

from . import _lib
from ._distances import METRIC_IDS, as_points, check_distance_range, validate_metric

_lib.lib.cuhc_trees_batched.restype = ctypes.c_int
_lib.lib.cuhc_trees_batched.argtypes = [
    ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int64), ctypes.c_int, ctypes.c_int,
    ctypes.c_int, ctypes.c_float, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_double),
    ctypes.POINTER(ctypes.c_float)]


def batched_trees(instances, min_samples, metric="euclidean", p=2.0):
    """[(Z_i, core_i)] for every instance, in input order. `min_samples` is
    one int per instance (0: single linkage, core_i all zero)."""
    validate_metric(metric, p)
    instances = [as_points(X, "instance") for X in instances]
    ks = [int(k) for k in min_samples]
    if len(ks) != len(instances):
        raise ValueError("one min_samples value per instance")
    for X, k in zip(instances, ks):
        if not 0 <= k <= X.shape[0]:
            raise ValueError(f"min_samples {k} outside [0, {X.shape[0]}]")
        check_distance_range(X, metric, p)
    out = [None] * len(instances)
    for d in sorted({X.shape[1] for X in instances}):
        group = [i for i, X in enumerate(instances) if X.shape[1] == d]
        sizes = np.array([instances[i].shape[0] for i in group], dtype=np.int64)
        offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        points = np.ascontiguousarray(np.concatenate([instances[i] for i in group]),
                                      dtype=np.float32)
        ranks = np.array([ks[i] for i in group], dtype=np.int32)
        trees = np.empty((int(offsets[-1]) - len(group), 4), dtype=np.float64)
        core = np.empty(int(offsets[-1]), dtype=np.float32)
        _lib.check(_lib.lib.cuhc_trees_batched(
            _lib.float_ptr(points), offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
            len(group), d, METRIC_IDS[metric], float(p),
            ranks.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), _lib.double_ptr(trees),
            _lib.float_ptr(core)))
        for j, i in enumerate(group):
            first = int(offsets[j]) - j
            out[i] = (trees[first:first + int(sizes[j]) - 1].copy(),
                      core[offsets[j]:offsets[j + 1]].copy())
    return out
