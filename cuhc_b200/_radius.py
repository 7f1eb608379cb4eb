"""Learned radius proposal for single-linkage Borůvka rounds (16 features).

A 19 -> 64 -> 64 -> 1 BF16 MLP (5,505 parameters) predicts, per point and
round, the log of the weight of its nearest other-component edge from the
point's scaled coordinates, log component size, round index and log of last
round's weight. The library caps each row's search at exp(prediction +
offset), certifies rows whose best edge lies inside the cap, and searches the
rest again without it, so trees never depend on the model. The model is off
until `set_radius_model` (or `load_radius_model`) is called.

Training (`train_radius_model`) logs exact rounds of given data sets
(`training_rows`) and fits the MLP with the library's GPU kernels (Adam on
mean squared error); `offset` is then chosen as a high quantile of the
residuals so most rows are certified.
"""

import ctypes
import pathlib

import numpy as np

from . import _lib

PARAMS = 5505
FEATURES = 19
DIMS = 16
MODEL_PATH = pathlib.Path(__file__).resolve().parent / "models" / "radius_d16.npz"

_f32 = ctypes.POINTER(ctypes.c_float)
_u64 = ctypes.POINTER(ctypes.c_uint64)
_i64 = ctypes.POINTER(ctypes.c_int64)
_L = _lib.lib
_L.cuhc_mlp_forward.restype = ctypes.c_int
_L.cuhc_mlp_forward.argtypes = [_f32, _f32, ctypes.c_int, _f32]
_L.cuhc_mlp_gradient.restype = ctypes.c_int
_L.cuhc_mlp_gradient.argtypes = [_f32, _f32, _f32, ctypes.c_int, _f32, _f32]
_L.cuhc_mlp_train.restype = ctypes.c_int
_L.cuhc_mlp_train.argtypes = [_f32, _f32, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                              ctypes.c_float, ctypes.c_uint64, _f32, _f32]
_L.cuhc_set_radius_model.restype = ctypes.c_int
_L.cuhc_set_radius_model.argtypes = [_f32, ctypes.c_float]
_L.cuhc_radius_stats.restype = ctypes.c_int
_L.cuhc_radius_stats.argtypes = [_u64, ctypes.c_int]
_L.cuhc_radius_training_rows.restype = ctypes.c_int
_L.cuhc_radius_training_rows.argtypes = [_f32, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_uint64, _f32, _f32, ctypes.c_int64, _i64]


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def mlp_forward(params, x):
    params, x = _f(params), _f(x)
    out = np.empty(len(x), np.float32)
    _lib.check(_L.cuhc_mlp_forward(_lib.float_ptr(params), _lib.float_ptr(x), len(x),
                                   _lib.float_ptr(out)))
    return out


def mlp_gradient(params, x, y):
    """(gradient of the mean squared error, mean squared error)."""
    params, x, y = _f(params), _f(x), _f(y)
    grad = np.empty(PARAMS, np.float32)
    loss = ctypes.c_float()
    _lib.check(_L.cuhc_mlp_gradient(_lib.float_ptr(params), _lib.float_ptr(x),
                                    _lib.float_ptr(y), len(y), _lib.float_ptr(grad),
                                    ctypes.byref(loss)))
    return grad, loss.value


def mlp_train(params, x, y, epochs=10, batch=1024, lr=1e-3, seed=0):
    """(trained params, per-epoch losses): Adam on the GPU."""
    params, x, y = _f(params).copy(), _f(x), _f(y)
    losses = np.empty(epochs, np.float32)
    _lib.check(_L.cuhc_mlp_train(_lib.float_ptr(x), _lib.float_ptr(y), len(y), epochs, batch,
                                 lr, seed, _lib.float_ptr(params), _lib.float_ptr(losses)))
    return params, losses


def training_rows(X, max_rows_per_round=20000, seed=0):
    """(features [m][19], targets [m]) logged from the exact rounds of X (n x 16)."""
    X = _f(X)
    if X.ndim != 2 or X.shape[1] != DIMS:
        raise ValueError(f"training rows need {DIMS} features")
    capacity = max_rows_per_round * 64
    feats = np.empty((capacity, FEATURES), np.float32)
    targets = np.empty(capacity, np.float32)
    rows = ctypes.c_int64()
    _lib.check(_L.cuhc_radius_training_rows(_lib.float_ptr(X), len(X), DIMS, max_rows_per_round,
                                            seed, _lib.float_ptr(feats),
                                            _lib.float_ptr(targets), capacity,
                                            ctypes.byref(rows)))
    m = min(rows.value, capacity)
    return feats[:m].copy(), targets[:m].copy()


def set_radius_model(params, offset=0.0):
    """Loads a model (5,505 floats); None switches the proposal off."""
    if params is None:
        _lib.check(_L.cuhc_set_radius_model(None, 0.0))
        return
    params = _f(params)
    if params.shape != (PARAMS,):
        raise ValueError(f"a radius model has {PARAMS} parameters")
    _lib.check(_L.cuhc_set_radius_model(_lib.float_ptr(params), float(offset)))


def load_radius_model(path=MODEL_PATH):
    """Loads the stored model (params, offset) and returns its metadata."""
    data = np.load(path, allow_pickle=False)
    set_radius_model(data["params"], float(data["offset"]))
    return {k: data[k] for k in data.files if k != "params"}


def radius_stats():
    """Since the last call: rows given a radius ('proposed'), rows settled by
    the capped pass ('certified'), tiles computed by the capped passes
    ('capped_tiles') and by the fallback passes ('fallback_tiles')."""
    out = (ctypes.c_uint64 * 4)()
    _lib.check(_L.cuhc_radius_stats(out, 4))
    return {"proposed": int(out[0]), "certified": int(out[1]), "capped_tiles": int(out[2]),
            "fallback_tiles": int(out[3])}


def init_params(seed=0):
    """He-initialised weights, zero biases (float32, the C layout:
    W1 [19][64], b1 [64], W2 [64][64], b2 [64], w3 [64], b3)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(PARAMS, np.float32)
    p[0:19 * 64] = rng.standard_normal(19 * 64) * np.sqrt(2.0 / 19)
    w2 = 19 * 64 + 64
    p[w2:w2 + 64 * 64] = rng.standard_normal(64 * 64) * np.sqrt(2.0 / 64)
    w3 = w2 + 64 * 64 + 64
    p[w3:w3 + 64] = rng.standard_normal(64) * np.sqrt(1.0 / 64)
    return p


def train_radius_model(datasets, epochs=20, batch=2048, lr=2e-3, quantile=0.95, seed=0,
                       max_rows_per_round=20000):
    """(params, offset, report): fits the MLP to rows logged from `datasets`
    (arrays n x 16); offset = the `quantile` of the training residuals, so
    that about that share of rows is certified by the first pass."""
    feats, targets = [], []
    for i, X in enumerate(datasets):
        f, t = training_rows(X, max_rows_per_round, seed + i)
        feats.append(f)
        targets.append(t)
    x = np.concatenate(feats)
    y = np.concatenate(targets)
    params = init_params(seed)
    params[-1] = float(np.mean(y))  # output bias at the mean target
    params, losses = mlp_train(params, x, y, epochs, batch, lr, seed)
    residual = y - mlp_forward(params, x)
    offset = float(np.quantile(residual, quantile))
    report = {"rows": len(y), "losses": losses, "offset": offset,
              "residual_std": float(np.std(residual))}
    return params, offset, report
