"""Surrogate-screened four-phonon scattering (no counterpart in the reference).

The reference evaluates the four-phonon rate of every irreducible mode exactly
(``src/Kappa/Src/main.f90:610-661``), which dominates its cost.  Here a small
network, trained on the device (``spring_mlp_*``) on exact rates from a coarse
mesh, predicts per-mode four-phonon rates from harmonic features; the
irreducible q0 blocks (all quartets of one q0) are ranked by the predicted
effect of their four-phonon scattering on kappa, the exact path
(``spring_linewidth4``) runs for the top fraction, and the prediction stands in
for the rest.  The exact path is both the fallback (fraction 1) and the measure
of the surrogate's error.

Features of a mode: omega (rad/ps), |group velocity| (m/s), its 3-phonon
scattering rate (2 x linewidth), branch index, |q| (1/A).  Target: log of the
four-phonon rate.  Features and targets are standardised with the training
set's mean and spread.
"""
from __future__ import annotations

import numpy as np

from .api import Context


def mode_features(omega, grp_vel, rate3, q_cart):
    """(n_q0 * Ndof, 5) features: omega, |v|, 3-phonon rate, branch index, |q|."""
    nq0, nd = omega.shape
    f = np.zeros((nq0, nd, 5))
    f[..., 0] = omega
    f[..., 1] = np.linalg.norm(grp_vel, axis=2)
    f[..., 2] = rate3
    f[..., 3] = np.arange(nd)[None, :]
    f[..., 4] = np.linalg.norm(q_cart, axis=1)[:, None]
    return f.reshape(-1, 5)


class Surrogate:
    """The device network with the standardisation of its training set."""

    def __init__(self, ctx: Context, seed: int = 0):
        self.ctx = ctx
        self.seed = seed
        self.xm = self.xs = None
        self.ym = self.ys = None

    def fit(self, X, log_rate, epochs=400, batch=64, lr=2e-3):
        X = np.asarray(X, np.float64)
        y = np.asarray(log_rate, np.float64)
        self.xm, self.xs = X.mean(axis=0), X.std(axis=0) + 1e-12
        self.ym, self.ys = y.mean(), y.std() + 1e-12
        self.ctx.mlp_init(self.seed)
        return self.ctx.mlp_train((X - self.xm) / self.xs, (y - self.ym) / self.ys, epochs=epochs,
                                  batch=min(batch, len(y)), lr=lr, seed=self.seed + 1)

    def predict(self, X, bf16=True):
        X = np.asarray(X, np.float64)
        z = self.ctx.mlp_predict((X - self.xm) / self.xs, bf16=bf16)
        return z.astype(np.float64) * self.ys + self.ym


def kappa_weight(omega, nbe, grp_vel, mult):
    """Per-mode weight of a scattering-time change in kappa: mult * omega^2 n (n + 1) |v|^2."""
    v2 = np.sum(grp_vel * grp_vel, axis=2)
    return mult[:, None] * omega ** 2 * nbe * (nbe + 1.0) * v2


def rank_blocks(rate3, rate4_pred, weight):
    """Irreducible q0 in decreasing order of the predicted kappa change of their 4-phonon rates,
    sum over branches of weight * (1/rate3 - 1/(rate3 + rate4))."""
    r3 = np.where(rate3 > 0, rate3, np.inf)
    d = weight * (1.0 / r3 - 1.0 / (r3 + np.maximum(rate4_pred, 0.0)))
    score = np.nansum(np.where(np.isfinite(d), d, 0.0), axis=1)
    return np.argsort(-score, kind="stable"), score


def screened_rates4(ctx: Context, rate4_pred, order, fraction, delta="gauss", sigma=0.3767, it=0):
    """Four-phonon rates (n_q0, Ndof) at temperature index ``it``: exact for the first
    ceil(fraction * n_q0) q0 of ``order``, the prediction elsewhere.  Returns (rates, exact mask)."""
    nq0 = rate4_pred.shape[0]
    k = int(np.ceil(fraction * nq0))
    exact = np.zeros(nq0, bool)
    rates = np.array(rate4_pred, np.float64)
    for i0 in order[:k]:
        rates[i0] = ctx.linewidth4(int(i0) + 1, 1, delta=delta, sigma=sigma)[it, 0]
        exact[i0] = True
    return rates, exact
