"""Metric ids, input validation and pairwise distances.

Same names, aliases, validation rules and messages as the reference's
python/cuhc/_distances.py (ids :8-18, as_points :28-36, float32 range guard
:42-72, pairwise_distances :75-134).
"""

import numpy as np

from . import _lib

# The C ABI's metric table; aliases are scikit-learn's names.
METRIC_IDS = {
    "euclidean": 0, "l2": 0,
    "sqeuclidean": 1,
    "manhattan": 2, "cityblock": 2, "l1": 2,
    "chebyshev": 3,
    "minkowski": 4,
    "cosine": 5,
}

FLOAT32_MAX = float(np.finfo(np.float32).max)


def validate_metric(metric, p):
    if metric not in METRIC_IDS:
        raise ValueError(f"unknown metric {metric!r}; choose from {sorted(METRIC_IDS)}")
    if METRIC_IDS[metric] == METRIC_IDS["minkowski"] and not p > 0:
        raise ValueError(f"the Minkowski order p must be positive, got {p!r}")


def as_points(array, name):
    """float32, C-contiguous, 2-D, non-empty and finite."""
    points = np.ascontiguousarray(array, dtype=np.float32)
    if points.ndim != 2:
        raise ValueError(f"{name} must be 2D (points x features); its shape is {points.shape}")
    if points.shape[0] == 0 or points.shape[1] == 0:
        raise ValueError(f"{name} must be non-empty; its shape is {points.shape}")
    if not np.isfinite(points).all():
        raise ValueError(f"{name} contains NaN or infinity")
    return points


class DevicePoints:
    """A float32, C-contiguous, 2-D array already in CUDA memory, seen
    through __cuda_array_interface__ (CuPy, PyTorch, Numba) or DLPack: the
    device entry points read it in place, with no host copy."""

    def __init__(self, owner, pointer, shape):
        self.owner, self.pointer, self.shape = owner, pointer, shape


def device_points(array, name):
    """DevicePoints for a CUDA array, None for anything else (host arrays).

    The array must be float32, C-contiguous, 2-D and non-empty; the work that
    produced it must be complete (PyTorch's and CuPy's current streams are
    synchronized here). NaN / infinity and the float32 range are not checked
    on the host for device arrays: non-finite distances still surface as the
    library's non-finite / disconnected errors."""
    owner = array
    cai = getattr(array, "__cuda_array_interface__", None)
    if cai is None and hasattr(array, "__dlpack__") and hasattr(array, "__dlpack_device__"):
        kind, _ = array.__dlpack_device__()
        if kind != 2:  # kDLCUDA
            return None
        import torch  # noqa: PLC0415 - DLPack objects are imported through torch
        owner = torch.utils.dlpack.from_dlpack(array)
        cai = owner.__cuda_array_interface__
    if cai is None:
        return None
    shape = tuple(int(x) for x in cai["shape"])
    if cai.get("typestr") != "<f4":
        raise ValueError(f"{name} on the GPU must be float32, got {cai.get('typestr')!r}")
    if len(shape) != 2:
        raise ValueError(f"{name} must be 2D (points x features); its shape is {shape}")
    if shape[0] == 0 or shape[1] == 0:
        raise ValueError(f"{name} must be non-empty; its shape is {shape}")
    strides = cai.get("strides")
    if strides is not None and tuple(strides) != (4 * shape[1], 4):
        raise ValueError(f"{name} on the GPU must be C-contiguous")
    _synchronize_producer(owner)
    return DevicePoints(owner, int(cai["data"][0]), shape)


def _synchronize_producer(owner):
    module = type(owner).__module__.split(".")[0]
    if module == "torch":
        import torch  # noqa: PLC0415
        torch.cuda.current_stream(owner.device).synchronize()
    elif module == "cupy":
        import cupy  # noqa: PLC0415
        cupy.cuda.get_current_stream().synchronize()


def _empty_like_device(owner, shape):
    """A float32 device array of `shape` from the input's own framework."""
    module = type(owner).__module__.split(".")[0]
    if module == "torch":
        import torch  # noqa: PLC0415
        out = torch.empty(shape, dtype=torch.float32, device=owner.device)
        return out, out.data_ptr()
    if module == "cupy":
        import cupy  # noqa: PLC0415
        out = cupy.empty(shape, dtype=cupy.float32)
        return out, out.data.ptr
    raise ValueError("pairwise_distances on device arrays needs PyTorch or CuPy arrays "
                     "(the output is allocated by the input's framework)")


def _distance_bound(spread, magnitude, metric, p):
    """Largest value any accumulated float32 distance of the data can take."""
    kind = METRIC_IDS[metric]
    if kind in (METRIC_IDS["euclidean"], METRIC_IDS["sqeuclidean"]):
        return float(np.sum(spread * spread))
    if kind == METRIC_IDS["manhattan"]:
        return float(np.sum(spread))
    if kind == METRIC_IDS["chebyshev"]:
        return float(np.max(spread))
    if kind == METRIC_IDS["minkowski"]:
        return float(np.sum(spread ** p))
    return float(np.sum(magnitude * magnitude))  # cosine accumulates squared norms


def check_distance_range(X, metric, p=2.0, Y=None, scale=1.0):
    """ValueError if a distance (times `scale`, e.g. Ward's cluster sizes or
    HDBSCAN's 1/alpha) could overflow float32. Each |x_k - y_k| is at most the
    feature's spread, so the bound is exact per feature and data far from the
    origin is fine."""
    values = X if Y is None else np.vstack([X, Y])
    with np.errstate(over="ignore", invalid="ignore"):
        spread = values.max(axis=0).astype(np.float64) - values.min(axis=0)
        magnitude = np.abs(values).max(axis=0).astype(np.float64)
        bound = _distance_bound(spread, magnitude, metric, p) * scale
    if not bound <= FLOAT32_MAX:
        raise ValueError(
            f"the data's range is too large for float32 {metric} distances (up to {bound:.3g}, "
            f"float32 holds {FLOAT32_MAX:.3g}); rescale the data")


def pairwise_distances(X, Y=None, metric="euclidean", p=2.0):
    """Distance of every row of X to every row of Y (Y defaults to X), in
    float32, like sklearn.metrics.pairwise_distances.

    Returns an (len(X), len(Y)) float32 array. Raises ValueError for unknown
    metrics, bad shapes, NaN/inf input or distances beyond float32.
    """
    validate_metric(metric, p)
    X_dev = device_points(X, "X")
    if X_dev is not None:
        return _pairwise_on_device(X_dev, Y, metric, p)
    X = as_points(X, "X")
    if Y is not None:
        Y = as_points(Y, "Y")
        if Y.shape[1] != X.shape[1]:
            raise ValueError("X and Y must have the same number of features, got "
                             f"{X.shape[1]} and {Y.shape[1]}")
    check_distance_range(X, metric, p, Y)
    rows_b = X.shape[0] if Y is None else Y.shape[0]
    out = np.empty((X.shape[0], rows_b), dtype=np.float32)
    _lib.check(_lib.lib.cuhc_pairwise_distances(
        _lib.float_ptr(X), X.shape[0], None if Y is None else _lib.float_ptr(Y), rows_b,
        X.shape[1], METRIC_IDS[metric], float(p), _lib.float_ptr(out)))
    return out


def _pairwise_on_device(X, Y, metric, p):
    """pairwise_distances of a device array: the output is a device array of
    the input's framework (PyTorch or CuPy)."""
    Y_dev = None if Y is None else device_points(Y, "Y")
    if Y is not None and Y_dev is None:
        raise ValueError("X and Y must both be device arrays or both host arrays")
    if Y_dev is not None and Y_dev.shape[1] != X.shape[1]:
        raise ValueError("X and Y must have the same number of features, got "
                         f"{X.shape[1]} and {Y_dev.shape[1]}")
    rows_b = X.shape[0] if Y_dev is None else Y_dev.shape[0]
    out, out_ptr = _empty_like_device(X.owner, (X.shape[0], rows_b))
    _lib.check(_lib.lib.cuhc_pairwise_distances_device(
        X.pointer, X.shape[0], None if Y_dev is None else Y_dev.pointer, rows_b, X.shape[1],
        METRIC_IDS[metric], float(p), out_ptr))
    return out
