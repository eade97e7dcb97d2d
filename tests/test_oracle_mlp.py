"""The network oracle's analytic gradient against central finite differences (CPU only)."""
import numpy as np

from oracle import mlp


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = rng.normal(0, 0.1, mlp.n_params())
    X = rng.normal(size=(17, 5))
    y = rng.normal(size=17)
    loss, g = mlp.loss_and_grad(p, X, y)
    idx = rng.choice(len(p), 60, replace=False)
    idx = np.concatenate([idx, [len(p) - 1, len(p) - 2]])  # include b4 and a W4 entry
    h = 1e-6
    for k in idx:
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (mlp.loss_and_grad(pp, X, y)[0] - mlp.loss_and_grad(pm, X, y)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g[k])) + 1e-8, (k, fd, g[k])
    assert mlp.n_params() == 33921
