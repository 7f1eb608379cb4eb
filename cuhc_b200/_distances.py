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
