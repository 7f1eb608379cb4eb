"""Oracle of the radius MLP (19 -> 64 -> 64 -> 1, ReLU, BF16): test
infrastructure only, never part of the product.

Plain NumPy restatement of the kernels' arithmetic (cuhc_b200/csrc/mlp.cu):
parameters, inputs and hidden activations rounded to BF16 (round to nearest
even), dot products accumulated in float64 (the kernels accumulate in FP32,
so outputs agree to FP32 rounding plus the rare BF16 activation that lands
on the other side of a rounding boundary), mean-squared-error gradients by
backpropagation. `finite_difference_gradient` checks the backpropagation
itself in float64 with no rounding. This model has no counterpart in the
reference; its tests pin it against this oracle.
"""

import numpy as np

IN, HIDDEN = 19, 64
W1, B1 = 0, IN * HIDDEN
W2 = B1 + HIDDEN
B2 = W2 + HIDDEN * HIDDEN
W3 = B2 + HIDDEN
B3 = W3 + HIDDEN
PARAMS = B3 + 1  # 5,505


def bf16(x):
    """Round float32 values to BF16 (nearest, ties to even), as float64."""
    a = np.asarray(x, dtype=np.float32)
    bits = a.view(np.uint32).astype(np.uint64)
    rounded = (bits + 0x7FFF + ((bits >> 16) & 1)) & 0xFFFF0000
    out = rounded.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out).astype(np.float64)


def unpack(params, rounding=True):
    p = bf16(params) if rounding else np.asarray(params, dtype=np.float64)
    return (p[W1:B1].reshape(IN, HIDDEN), p[B1:W2], p[W2:B2].reshape(HIDDEN, HIDDEN), p[B2:W3],
            p[W3:B3], p[B3])


def forward(params, x, rounding=True):
    """(out, h1, h2) for samples x [m][19]."""
    r = bf16 if rounding else (lambda v: np.asarray(v, dtype=np.float64))
    w1, b1, w2, b2, w3, b3 = unpack(params, rounding)
    xin = r(x)
    h1 = r(np.maximum(xin @ w1 + b1, 0.0).astype(np.float32) if rounding else
           np.maximum(xin @ w1 + b1, 0.0))
    h2 = r(np.maximum(h1 @ w2 + b2, 0.0).astype(np.float32) if rounding else
           np.maximum(h1 @ w2 + b2, 0.0))
    return h2 @ w3 + b3, h1, h2, xin


def gradient(params, x, y, rounding=True):
    """(d mean((out - y)^2) / d params, mean squared error)."""
    _, _, w2, _, w3, _ = unpack(params, rounding)
    out, h1, h2, xin = forward(params, x, rounding)
    m = len(y)
    err = out - np.asarray(y, dtype=np.float64)
    dout = 2.0 * err / m
    d2 = (h2 > 0) * dout[:, None] * w3[None, :]
    d1 = (h1 > 0) * (d2 @ w2.T)
    g = np.zeros(PARAMS)
    g[W1:B1] = (xin.T @ d1).ravel()
    g[B1:W2] = d1.sum(axis=0)
    g[W2:B2] = (h1.T @ d2).ravel()
    g[B2:W3] = d2.sum(axis=0)
    g[W3:B3] = h2.T @ dout
    g[B3] = dout.sum()
    return g, float(np.mean(err ** 2))


def finite_difference_gradient(params, x, y, indices, eps=1e-6):
    """Central differences of the unrounded float64 loss at `indices`."""
    p = np.asarray(params, dtype=np.float64)
    out = []
    for i in indices:
        up, down = p.copy(), p.copy()
        up[i] += eps
        down[i] -= eps
        lu = np.mean((forward(up, x, False)[0] - y) ** 2)
        ld = np.mean((forward(down, x, False)[0] - y) ** 2)
        out.append((lu - ld) / (2 * eps))
    return np.array(out)


def init_params(seed=0):
    """He-initialised weights, zero biases (float32)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(PARAMS, dtype=np.float32)
    p[W1:B1] = rng.standard_normal(IN * HIDDEN) * np.sqrt(2.0 / IN)
    p[W2:B2] = rng.standard_normal(HIDDEN * HIDDEN) * np.sqrt(2.0 / HIDDEN)
    p[W3:B3] = rng.standard_normal(HIDDEN) * np.sqrt(1.0 / HIDDEN)
    return p
