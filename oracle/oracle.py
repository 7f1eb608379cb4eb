"""ctypes wrapper of the CPU oracle (oracle.c). Test infrastructure only: the
checker for tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg.

Every function takes float32 C-contiguous NumPy arrays and returns NumPy
arrays; status codes follow the reference's C API (-2 shape, -5
disconnected, ...).
"""

import ctypes
import pathlib

import numpy as np

_HERE = pathlib.Path(__file__).resolve().parent
_LIB_PATH = _HERE / "liboracle.so"
_REF_PATH = _HERE / "_ref" / "libcuhc.so"

_f32 = ctypes.POINTER(ctypes.c_float)
_f64 = ctypes.POINTER(ctypes.c_double)
_i32 = ctypes.POINTER(ctypes.c_int)
_i64 = ctypes.POINTER(ctypes.c_int64)
_u64 = ctypes.POINTER(ctypes.c_uint64)

METRICS = {"euclidean": 0, "sqeuclidean": 1, "manhattan": 2, "chebyshev": 3, "minkowski": 4,
           "cosine": 5}

_lib = None


def lib():
    """The oracle library, built on first use if this machine can compile it."""
    global _lib
    if _lib is None:
        if not _LIB_PATH.exists():
            from oracle.build import build_oracle  # noqa: PLC0415
            build_oracle()
        _lib = ctypes.CDLL(str(_LIB_PATH))
        _declare(_lib)
    return _lib


def _declare(L):
    L.orc_set_threads.argtypes = [ctypes.c_int]
    L.orc_get_threads.restype = ctypes.c_int
    L.orc_pairwise.argtypes = [_f32, ctypes.c_int, _f32, ctypes.c_int, ctypes.c_int,
                               ctypes.c_int, ctypes.c_float, _f32]
    L.orc_core_distances_rows.argtypes = [_f32, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, _f32]
    L.orc_nearest_other_component.argtypes = [_f32, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_float, _f32, ctypes.c_float, _i32, _u64]
    L.orc_mst.argtypes = [_f32, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float, _f32,
                          ctypes.c_float, _i32, _i32, _f32]
    L.orc_tree_from_mst.argtypes = [_i32, _i32, _f32, ctypes.c_int, _f64]
    L.orc_single_linkage.argtypes = [_f32, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_float, _f64]
    L.orc_hdbscan_tree.argtypes = [_f32, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.c_float, ctypes.c_int, ctypes.c_float, _f64, _f32]
    L.orc_condense_tree.restype = ctypes.c_int64
    L.orc_condense_tree.argtypes = [_f64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                    _i64, _i64, _f64, _i64]


def _p(array, kind):
    return None if array is None else array.ctypes.data_as(kind)


def _points(X):
    return np.ascontiguousarray(X, dtype=np.float32)


def _check(status):
    if status != 0:
        raise RuntimeError(f"oracle status {status}")


def set_threads(threads):
    lib().orc_set_threads(int(threads))


def threads():
    return lib().orc_get_threads()


def pairwise(X, Y=None, metric="euclidean", p=2.0):
    X = _points(X)
    Y = None if Y is None else _points(Y)
    nB = X.shape[0] if Y is None else Y.shape[0]
    out = np.empty((X.shape[0], nB), np.float32)
    _check(lib().orc_pairwise(_p(X, _f32), X.shape[0], _p(Y, _f32), nB, X.shape[1],
                              METRICS[metric], p, _p(out, _f32)))
    return out


def core_distances(X, k, metric="euclidean", p=2.0, rows=None):
    X = _points(X)
    begin, end = (0, X.shape[0]) if rows is None else rows
    core = np.empty(end - begin, np.float32)
    _check(lib().orc_core_distances_rows(_p(X, _f32), X.shape[0], X.shape[1], METRICS[metric], p,
                                         int(k), begin, end, _p(core, _f32)))
    return core


def nearest_other_component(X, component, metric="euclidean", p=2.0, core=None, alpha=1.0):
    X = _points(X)
    component = np.ascontiguousarray(component, np.int32)
    core = None if core is None else np.ascontiguousarray(core, np.float32)
    nearest = np.empty(X.shape[0], np.uint64)
    _check(lib().orc_nearest_other_component(_p(X, _f32), X.shape[0], X.shape[1],
                                             METRICS[metric], p, _p(core, _f32), alpha,
                                             _p(component, _i32), _p(nearest, _u64)))
    return nearest


def mst(X, metric="euclidean", p=2.0, core=None, alpha=1.0):
    """(u, v, w) of the unique MST under the (weight, min, max) edge order."""
    X = _points(X)
    n = X.shape[0]
    u, v = np.empty(max(n - 1, 0), np.int32), np.empty(max(n - 1, 0), np.int32)
    w = np.empty(max(n - 1, 0), np.float32)
    core = None if core is None else np.ascontiguousarray(core, np.float32)
    _check(lib().orc_mst(_p(X, _f32), n, X.shape[1], METRICS[metric], p, _p(core, _f32), alpha,
                         _p(u, _i32), _p(v, _i32), _p(w, _f32)))
    return u, v, w


def tree_from_mst(u, v, w, n):
    Z = np.empty((max(n - 1, 0), 4), np.float64)
    u, v = np.ascontiguousarray(u, np.int32), np.ascontiguousarray(v, np.int32)
    w = np.ascontiguousarray(w, np.float32)
    lib().orc_tree_from_mst(_p(u, _i32), _p(v, _i32), _p(w, _f32), n, _p(Z, _f64))
    return Z


def single_linkage(X, metric="euclidean", p=2.0):
    X = _points(X)
    Z = np.empty((max(X.shape[0] - 1, 0), 4), np.float64)
    _check(lib().orc_single_linkage(_p(X, _f32), X.shape[0], X.shape[1], METRICS[metric], p,
                                    _p(Z, _f64)))
    return Z


def hdbscan_tree(X, min_samples, metric="euclidean", p=2.0, alpha=1.0):
    X = _points(X)
    n = X.shape[0]
    Z = np.empty((max(n - 1, 0), 4), np.float64)
    core = np.empty(n, np.float32)
    _check(lib().orc_hdbscan_tree(_p(X, _f32), n, X.shape[1], METRICS[metric], p,
                                  int(min_samples), alpha, _p(Z, _f64), _p(core, _f32)))
    return Z, core


def condense_tree(Z, min_cluster_size):
    Z = np.ascontiguousarray(Z, np.float64)
    n = len(Z) + 1
    capacity = n + 2 * (n // max(int(min_cluster_size), 1)) + 2
    out = [np.empty(capacity, np.int64), np.empty(capacity, np.int64),
           np.empty(capacity, np.float64), np.empty(capacity, np.int64)]
    rows = lib().orc_condense_tree(_p(Z, _f64), n, int(min_cluster_size), capacity,
                                   _p(out[0], _i64), _p(out[1], _i64), _p(out[2], _f64),
                                   _p(out[3], _i64))
    if rows < 0:
        raise RuntimeError(f"condensed tree needs {-rows} rows")
    return tuple(a[:rows] for a in out)


# ---- the reference library itself (oracle/_ref), when it was built -------

def reference_available():
    return _REF_PATH.exists()


_ref = None


def reference():
    """ctypes handle of the reference libcuhc.so (oracle/_ref), declared with
    the reference's own signatures (its python/cuhc/_lib.py:19-91)."""
    global _ref
    if _ref is None:
        R = ctypes.CDLL(str(_REF_PATH))
        R.cuhc_linkage.argtypes = [_f32, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                   ctypes.c_int, ctypes.c_int, _f64]
        R.cuhc_hdbscan_tree.argtypes = [_f32, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_float, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                        _f64, _f32]
        R.cuhc_ward_rnn_with_options.argtypes = [_f32, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                                 ctypes.c_int, ctypes.c_int, _f64]
        R.cuhc_pairwise_distances.argtypes = [_f32, ctypes.c_int, _f32, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_int, ctypes.c_float, _f32]
        R.cuhc_condense_tree.restype = ctypes.c_int64
        R.cuhc_condense_tree.argtypes = [_f64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                         _i64, _i64, _f64, _i64]
        R.cuhc_set_pruning.argtypes = [ctypes.c_int]
        R.cuhc_prune_stats.argtypes = [_u64, _u64]
        R.cuhc_error_string.restype = ctypes.c_char_p
        R.cuhc_error_string.argtypes = [ctypes.c_int]
        _ref = R
    return _ref


def reference_condense_tree(Z, min_cluster_size):
    """The reference's C++ condensing (CPU only, runs without a GPU)."""
    R = reference()
    Z = np.ascontiguousarray(Z, np.float64)
    n = len(Z) + 1
    capacity = n + 2 * (n // max(int(min_cluster_size), 1)) + 2
    out = [np.empty(capacity, np.int64), np.empty(capacity, np.int64),
           np.empty(capacity, np.float64), np.empty(capacity, np.int64)]
    rows = R.cuhc_condense_tree(_p(Z, _f64), n, int(min_cluster_size), capacity,
                                _p(out[0], _i64), _p(out[1], _i64), _p(out[2], _f64),
                                _p(out[3], _i64))
    if rows < 0:
        raise RuntimeError(f"condensed tree needs {-rows} rows")
    return tuple(a[:rows] for a in out)


def reference_check(status):
    if status != 0:
        raise RuntimeError(f"reference: {reference().cuhc_error_string(status).decode()} "
                           f"(code {status})")


PRUNE_MODES = {"auto": 0, "always": 1, "never": 2}


def reference_linkage(X, method="single", algorithm="mst", metric="euclidean", p=2.0,
                      pruning="never"):
    """The reference's cuhc_linkage (GPU), with its pruning mode set first."""
    R = reference()
    linkages = {"single": 0, "complete": 1, "average": 2, "ward": 3}
    algorithms = {"dense": 0, "mst": 1, "nn_chain": 2, "rnn": 3}
    X = _points(X)
    n = X.shape[0]
    Z = np.empty((max(n - 1, 0), 4), np.float64)
    reference_check(R.cuhc_set_pruning(PRUNE_MODES[pruning]))
    reference_check(R.cuhc_linkage(_p(X, _f32), n, X.shape[1], METRICS[metric], p,
                                   linkages[method], algorithms[algorithm], _p(Z, _f64)))
    return Z


def reference_hdbscan_tree(X, min_samples, metric="euclidean", p=2.0, alpha=1.0,
                           core_method=0, pruning="never"):
    R = reference()
    X = _points(X)
    n = X.shape[0]
    Z = np.empty((max(n - 1, 0), 4), np.float64)
    core = np.empty(n, np.float32)
    reference_check(R.cuhc_set_pruning(PRUNE_MODES[pruning]))
    reference_check(R.cuhc_hdbscan_tree(_p(X, _f32), n, X.shape[1], METRICS[metric], p,
                                        int(min_samples), alpha, core_method, _p(Z, _f64),
                                        _p(core, _f32)))
    return Z, core
