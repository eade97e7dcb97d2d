"""The surrogate network's device kernels (through the C ABI) against the numpy oracle: forward pass,
gradient, training progress and BF16 inference."""
import numpy as np
import pytest

from oracle import mlp
from spring_b200.api import Context

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = Context(2, (4, 4, 4), 1)
    c.mlp_init(seed=11)
    yield c
    c.close()


def _data(n, seed=5):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, 5)).astype(np.float32)
    y = (np.sin(X[:, 0]) + 0.5 * X[:, 1] * X[:, 2] - 0.3 * X[:, 3] ** 2 + 0.1 * X[:, 4]).astype(np.float32)
    return X, y


def test_predict_matches_oracle(ctx):
    X, _ = _data(300)
    p = ctx.mlp_params().astype(np.float64)
    ref, _ = mlp.forward(p, X)
    out = ctx.mlp_predict(X)
    np.testing.assert_allclose(out, ref, rtol=1e-4, atol=1e-5 * np.abs(ref).max())
    out16 = ctx.mlp_predict(X, bf16=True)
    assert np.abs(out16 - ref).max() < 3e-2 * np.abs(ref).max()


def test_gradient_matches_oracle(ctx):
    X, y = _data(257)
    p = ctx.mlp_params().astype(np.float64)
    loss_ref, g_ref = mlp.loss_and_grad(p, X, y)
    loss, g = ctx.mlp_loss_grad(X, y)
    assert abs(loss - loss_ref) <= 1e-5 * loss_ref
    np.testing.assert_allclose(g, g_ref, rtol=1e-3, atol=1e-5 * np.abs(g_ref).max())


def test_training_reduces_loss_and_generalises(ctx):
    X, y = _data(4096)
    Xt, yt = _data(1024, seed=9)
    ctx.mlp_init(seed=2)
    before = float(np.mean((ctx.mlp_predict(Xt) - yt) ** 2))
    hist = ctx.mlp_train(X, y, epochs=60, batch=256, lr=2e-3, seed=4)
    after = float(np.mean((ctx.mlp_predict(Xt) - yt) ** 2))
    assert hist[-1] < 0.2 * hist[0]
    assert after < 0.1 * before
    # the trained parameters reproduce on the oracle
    p = ctx.mlp_params().astype(np.float64)
    ref, _ = mlp.forward(p, Xt)
    np.testing.assert_allclose(ctx.mlp_predict(Xt), ref, rtol=1e-3, atol=1e-4)


def test_set_params_round_trip(ctx):
    p = np.random.default_rng(1).normal(0, 0.05, mlp.n_params()).astype(np.float32)
    ctx.mlp_set_params(p)
    np.testing.assert_array_equal(ctx.mlp_params(), p)
