"""CPU: the radius MLP's oracle (backpropagation against finite differences,
BF16 rounding) and the host side of the radius API."""

import numpy as np
import pytest

from cuhc_b200 import _radius
from oracle import mlp


def test_oracle_backprop_matches_finite_differences():
    p = mlp.init_params(3).astype(np.float64)
    rng = np.random.default_rng(1)
    x, y = rng.standard_normal((40, 19)), rng.standard_normal(40)
    g, _ = mlp.gradient(p, x, y, rounding=False)
    idx = [0, 500, mlp.B1 + 7, mlp.W2 + 1000, mlp.B2 + 3, mlp.W3 + 11, mlp.B3]
    fd = mlp.finite_difference_gradient(p, x, y, idx)
    np.testing.assert_allclose(g[idx], fd, rtol=1e-5, atol=1e-9)


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.005859375, 3.14159, -2.5e-3, 0.0], np.float32)
    out = mlp.bf16(v)
    np.testing.assert_array_equal(out[:3], [1.0, 1.0, 1.0078125])
    assert np.all(np.abs(out - v) <= np.abs(v) * 2.0 ** -8)


def test_layouts_agree():
    assert mlp.PARAMS == _radius.PARAMS == 5505
    p = _radius.init_params(0)
    assert p.shape == (5505,)
    assert np.all(p[mlp.B1:mlp.W2] == 0) and np.all(p[mlp.B2:mlp.W3] == 0) and p[mlp.B3] == 0


def test_model_shape_checked():
    with pytest.raises(ValueError):
        _radius.set_radius_model(np.zeros(10, np.float32))
    with pytest.raises(ValueError):
        _radius.training_rows(np.zeros((10, 3), np.float32))
