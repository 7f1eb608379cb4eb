"""ctypes binding of libcuhc.so (built in-tree by cuhc_b200/build.py).

The declarations mirror the C ABI in include/cuhc.h, which keeps the
reference's eight entry points (shangar21/cuhc python/cuhc/_lib.py:19-91)
unchanged and adds device-pointer variants and pass statistics. Importing
fails loudly when the library is missing: there is no CPU fallback.
"""

import ctypes
import pathlib

_LIB_PATH = pathlib.Path(__file__).resolve().parent / "libcuhc.so"

if not _LIB_PATH.exists():
    raise ImportError(
        f"{_LIB_PATH} is missing; build it with `python cuhc_b200/build.py` "
        "(nvcc for sm_100a). cuhc_b200 has no CPU fallback.")

lib = ctypes.CDLL(str(_LIB_PATH))

_f32 = ctypes.POINTER(ctypes.c_float)
_f64 = ctypes.POINTER(ctypes.c_double)
_i64 = ctypes.POINTER(ctypes.c_int64)
_u64 = ctypes.POINTER(ctypes.c_uint64)
_int, _float = ctypes.c_int, ctypes.c_float

lib.cuhc_pairwise_distances.restype = _int
lib.cuhc_pairwise_distances.argtypes = [_f32, _int, _f32, _int, _int, _int, _float, _f32]
lib.cuhc_linkage.restype = _int
lib.cuhc_linkage.argtypes = [_f32, _int, _int, _int, _float, _int, _int, _f64]
lib.cuhc_ward_rnn_with_options.restype = _int
lib.cuhc_ward_rnn_with_options.argtypes = [_f32, _int, _int, _float, _int, _int, _f64]
lib.cuhc_hdbscan_tree.restype = _int
lib.cuhc_hdbscan_tree.argtypes = [_f32, _int, _int, _int, _float, _int, _float, _int, _f64, _f32]
lib.cuhc_condense_tree.restype = ctypes.c_int64
lib.cuhc_condense_tree.argtypes = [_f64, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                   _i64, _i64, _f64, _i64]
lib.cuhc_set_pruning.restype = _int
lib.cuhc_set_pruning.argtypes = [_int]
lib.cuhc_prune_stats.restype = None
lib.cuhc_prune_stats.argtypes = [_u64, _u64]
lib.cuhc_error_string.restype = ctypes.c_char_p
lib.cuhc_error_string.argtypes = [_int]

# Additions (no counterpart in the reference).
lib.cuhc_linkage_device.restype = _int
lib.cuhc_linkage_device.argtypes = [ctypes.c_void_p, _int, _int, _int, _float, _int, _int, _f64]
lib.cuhc_hdbscan_tree_device.restype = _int
lib.cuhc_hdbscan_tree_device.argtypes = [ctypes.c_void_p, _int, _int, _int, _float, _int, _float,
                                         _int, _f64, _f32]
lib.cuhc_pairwise_distances_device.restype = _int
lib.cuhc_pairwise_distances_device.argtypes = [ctypes.c_void_p, _int, ctypes.c_void_p, _int, _int,
                                               _int, _float, ctypes.c_void_p]
lib.cuhc_pass_stats.restype = _int
lib.cuhc_pass_stats.argtypes = [_u64, _int]

lib.cuhc_hdbscan_labels.restype = _int
lib.cuhc_hdbscan_labels.argtypes = [_f64, ctypes.c_int64, ctypes.c_int64, _int, _int,
                                    ctypes.c_double, ctypes.c_int64, _i64, _f64]
lib.cuhc_screen_counters.restype = _int
lib.cuhc_screen_counters.argtypes = [ctypes.POINTER(ctypes.c_uint64), _int]
lib.cuhc_set_screen.restype = _int
lib.cuhc_set_screen.argtypes = [_int]
lib.cuhc_launch_count.restype = ctypes.c_uint64
lib.cuhc_launch_count.argtypes = []
lib.cuhc_set_timing.restype = _int
lib.cuhc_set_timing.argtypes = [_int]
lib.cuhc_kernel_timing.restype = _int
lib.cuhc_kernel_timing.argtypes = [_f64, _u64, _u64, _int]
lib.cuhc_set_screen_audit.restype = _int
lib.cuhc_set_screen_audit.argtypes = [_int]
lib.cuhc_screen_audit.restype = _int
lib.cuhc_screen_audit.argtypes = [_f64, _int]
lib.cuhc_screen_shape.restype = _int
lib.cuhc_screen_shape.argtypes = [ctypes.POINTER(_int), ctypes.POINTER(_int)]
lib.cuhc_wait_selftest.restype = _int
lib.cuhc_wait_selftest.argtypes = [_int, _int, _int]

PRUNE_MODES = {"auto": 0, "always": 1, "never": 2}
SCREEN_MODES = {"auto": 0, "on": 1, "off": 2}
# Pass kinds of cuhc_kernel_timing.
TIMER_KINDS = ("knn_pass", "nearest_pass", "screen_pass", "screen_knn_pass")
# cudaErrorMemoryAllocation, reported by the dense path as MemoryError.
CUDA_ERROR_OUT_OF_MEMORY = 2


def check(status):
    """RuntimeError with the library's message for a non-zero status."""
    if status != 0:
        raise RuntimeError(f"cuhc: {lib.cuhc_error_string(status).decode()} (code {status})")


def float_ptr(array):
    return array.ctypes.data_as(_f32)


def double_ptr(array):
    return array.ctypes.data_as(_f64)


def int64_ptr(array):
    return array.ctypes.data_as(_i64)


def set_pruning(mode):
    """Spatial pruning of the matrix-free paths: "auto", "always" or "never".
    Results are identical in every mode; only the time changes."""
    check(lib.cuhc_set_pruning(PRUNE_MODES[mode]))


def set_screen(mode):
    """Tensor-core screening of the all-pairs passes: "auto" (on for euclidean
    and sqeuclidean up to 32 features), "on" or "off". Results are identical
    in every mode; only the time changes."""
    check(lib.cuhc_set_screen(SCREEN_MODES[mode]))


SCREEN_COUNTERS = ("rechecks", "slow_rows", "indicator_tiles", "masked_tiles", "prefiltered")


def screen_counters():
    """Screened-pass counters since the last call (counted while timing is
    on): exact rechecks, row visits that took the exact path, tiles whose
    components were excluded by indicator slots, tiles masked in the
    epilogue, candidate tiles no row of the block needed."""
    out = (ctypes.c_uint64 * len(SCREEN_COUNTERS))()
    check(lib.cuhc_screen_counters(out, len(SCREEN_COUNTERS)))
    return dict(zip(SCREEN_COUNTERS, (int(x) for x in out)))


def prune_stats():
    """(tiles computed, tiles in all passes) since the last call; resets."""
    computed, total = ctypes.c_uint64(), ctypes.c_uint64()
    lib.cuhc_prune_stats(ctypes.byref(computed), ctypes.byref(total))
    return computed.value, total.value


def pass_stats():
    """Cumulative (tiles computed, tiles total, passes, Borůvka rounds)."""
    out = (ctypes.c_uint64 * 4)()
    lib.cuhc_pass_stats(out, 4)
    return tuple(int(x) for x in out)


def launch_count():
    """Kernel launches of libcuhc.so since it was loaded."""
    return int(lib.cuhc_launch_count())


def set_timing(on):
    """Per-pass CUDA-event timing on the launching stream (off by default)."""
    check(lib.cuhc_set_timing(1 if on else 0))


def kernel_timing():
    """{kind: (device ms, launches, tiles computed)} since the last call; resets."""
    ms = (ctypes.c_double * 4)()
    launches, tiles = (ctypes.c_uint64 * 4)(), (ctypes.c_uint64 * 4)()
    check(lib.cuhc_kernel_timing(ms, launches, tiles, 4))
    return {TIMER_KINDS[i]: (ms[i], int(launches[i]), int(tiles[i])) for i in range(4)}


AUDIT_FIELDS = ("pairs", "violations", "min_slack", "max_bound_gap_rel_norms", "max_bound_gap_abs",
                "max_exact_abs", "max_exact_rel")


def set_screen_audit(on):
    """Audit of the tensor-core screen (off by default): every pair of every
    screened tile is also checked against the reference FP32 distance and an
    FP64 recomputation. Results never change; audited passes are slower."""
    check(lib.cuhc_set_screen_audit(1 if on else 0))


def screen_audit():
    """Audit results since the last call (resets): pairs audited,
    violations of the screen's guarantee D' <= s (must be 0), the smallest
    slack (s - D') / (e (|x|^2 + |y|^2)) (>= 0 required; about 0.5 or more
    means the modelled error bound holds with room), the largest gap of the
    screened bound below the FP64 value (relative to the norms, and
    absolute), and the largest absolute / relative error of the reference
    FP32 squared distance against FP64. NaN where nothing was observed."""
    out = (ctypes.c_double * len(AUDIT_FIELDS))()
    check(lib.cuhc_screen_audit(out, len(AUDIT_FIELDS)))
    values = [float(x) for x in out]
    values[0], values[1] = int(values[0]), int(values[1])
    return dict(zip(AUDIT_FIELDS, values))


def screen_shape():
    """(ring slots, copy lead) the shape tuner chose for the latest screened
    k-NN pass ((0, 0) before any)."""
    stages, lead = _int(), _int()
    check(lib.cuhc_screen_shape(ctypes.byref(stages), ctypes.byref(lead)))
    return stages.value, lead.value
