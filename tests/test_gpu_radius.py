"""GPU: the radius MLP's kernels against the NumPy oracle (forward, mean
squared error gradient), GPU training, and the radius proposal in Borůvka:
trees are identical with and without a model whatever the model predicts
(certification and fallback), and the counters add up."""

import numpy as np
import pytest

import cuhc_b200 as C
from cuhc_b200 import _lib, _radius
from cuhc_b200.train_radius import make_anisotropic_blobs
from oracle import mlp
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture
def no_model():
    yield
    C.set_radius_model(None)


def _samples(m, seed=0):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((m, 19)).astype(np.float32), rng.standard_normal(m).astype(np.float32)


def test_forward_matches_oracle():
    p = _radius.init_params(5)
    x, _ = _samples(3000)
    got = _radius.mlp_forward(p, x)
    ref = mlp.forward(p, x)[0]
    # FP32 accumulation against float64, plus rare BF16 activations rounded
    # the other way: a BF16-level tolerance.
    np.testing.assert_allclose(got, ref, rtol=2e-2, atol=2e-2 * np.abs(ref).mean())


def test_gradient_matches_oracle():
    p = _radius.init_params(6)
    x, y = _samples(1000, 1)
    g, loss = _radius.mlp_gradient(p, x, y)
    g_ref, loss_ref = mlp.gradient(p, x, y)
    assert abs(loss - loss_ref) <= 1e-2 * loss_ref
    assert np.linalg.norm(g - g_ref) <= 2e-2 * np.linalg.norm(g_ref)
    for part in (slice(mlp.W1, mlp.B1), slice(mlp.W2, mlp.B2), slice(mlp.W3, mlp.B3)):
        assert np.linalg.norm(g[part] - g_ref[part]) <= 3e-2 * np.linalg.norm(g_ref[part])


def test_training_reduces_loss():
    rng = np.random.default_rng(2)
    x = rng.uniform(-1, 1, (20000, 19)).astype(np.float32)
    y = (np.sin(2 * x[:, 0]) + 0.5 * x[:, 1] * x[:, 2]).astype(np.float32)
    p0 = _radius.init_params(0)
    p, losses = _radius.mlp_train(p0, x, y, epochs=8, batch=512, lr=2e-3)
    assert losses[-1] < 0.25 * losses[0]
    _, l_end = _radius.mlp_gradient(p, x, y)
    assert l_end < 0.3 * np.mean((y - y.mean()) ** 2) + 1e-3


def test_training_rows():
    X = make_anisotropic_blobs(12, 20000)
    f, t = _radius.training_rows(X, max_rows_per_round=500, seed=1)
    assert f.shape[1] == 19 and len(f) == len(t) and 500 <= len(t) <= 500 * 64
    assert np.all(np.isfinite(f)) and np.all(np.isfinite(t))
    assert np.all(np.abs(f[:, :16]) <= 1.0 + 1e-6)        # scaled coordinates
    assert set(np.unique(f[:, 17])) <= set(range(64))      # round index


@pytest.mark.parametrize("offset", [-30.0, -1.0, 0.0, 1.0, 30.0])
def test_trees_identical_with_any_model(no_model, offset):
    X = make_anisotropic_blobs(7, 30000)
    ref = O.single_linkage(X)
    rng = np.random.default_rng(4)
    x = rng.uniform(-1, 1, (4000, 19)).astype(np.float32)
    y = rng.normal(-1.0, 0.5, 4000).astype(np.float32)
    p, _ = _radius.mlp_train(_radius.init_params(1), x, y, epochs=2, batch=512)
    C.set_radius_model(p, offset)
    C.radius_stats()
    Z = C.linkage(X, "single")
    stats = C.radius_stats()
    np.testing.assert_array_equal(Z, ref)
    assert stats["proposed"] >= len(X) and 0 <= stats["certified"] <= stats["proposed"]
    if offset == -30.0:
        assert stats["certified"] == 0      # radii ~0: every row falls back
    if offset == 30.0:
        assert stats["certified"] > 0


def test_other_dimensions_do_not_use_the_model(no_model):
    C.set_radius_model(_radius.init_params(2), 0.0)
    C.radius_stats()
    X = make_anisotropic_blobs(8, 5000)[:, :8].copy()
    np.testing.assert_array_equal(C.linkage(X, "single"), O.single_linkage(X))
    assert C.radius_stats()["proposed"] == 0


def test_shipped_model_gain_and_cost(no_model):
    """What the trained network gains, measured on 500,000 points of the
    4,000,000 x 16 recipe (seed 3): the same tree with and without it; with
    it, the capped first passes of the rounds compute fewer tiles than the
    whole search without it computes (the gain: rows stop at their proposed
    radius), and the uncertified rows' fallback passes cost the rest (the
    cost, which decides whether the proposal pays)."""
    X = make_anisotropic_blobs(3, 500_000)
    _lib.set_timing(True)
    try:
        _lib.kernel_timing()
        Z_plain = C.linkage(X, "single")
        tiles_without = _lib.kernel_timing()["screen_pass"][2]
        C.load_radius_model()
        C.radius_stats()
        Z_model = C.linkage(X, "single")
        stats = C.radius_stats()
    finally:
        _lib.set_timing(False)
        C.set_radius_model(None)
    np.testing.assert_array_equal(Z_model, Z_plain)
    assert stats["certified"] > 0.5 * stats["proposed"], stats
    assert 0 < stats["capped_tiles"] < tiles_without, (stats, tiles_without)
    assert stats["fallback_tiles"] > 0, stats
    print(f"tiles without the model {tiles_without:,}; with it: capped passes "
          f"{stats['capped_tiles']:,}, fallback passes {stats['fallback_tiles']:,}; "
          f"certified {stats['certified'] / stats['proposed']:.3f}")
