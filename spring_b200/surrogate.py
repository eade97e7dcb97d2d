"""Surrogate-screened four-phonon scattering (no counterpart in the reference).

The reference evaluates the four-phonon rate of every irreducible mode exactly
(``src/Kappa/Src/main.f90:610-661``), which dominates its cost.  Here a small
network, trained on the device (``spring_mlp_*``) on exact rates from a coarse
mesh, predicts per-mode four-phonon rates from harmonic features.  The quartet
sum of a q0 is cut into blocks by the branch s0 it scatters (the tensor-core V4
computes one block per pair of its (s0, s1) chunks, so the exact work of a block
is one sixth of the q0's); the blocks are ranked by the predicted effect of
their rate on kappa, weighted up where the network is uncertain (the spread of
an ensemble), exact V4 (``spring_linewidth4_modes``) runs for the top fraction,
and the prediction stands in for the rest.  The exact path is both the fallback
(fraction 1) and the measure of the surrogate's error.

Features of a mode: omega (rad/ps), |group velocity| (m/s), its 3-phonon
scattering rate (2 x linewidth), branch index, |q| (1/A).  Target: log of the
four-phonon rate.  Features and targets are standardised with the training
set's mean and spread.

``PowerLaw`` is the network-free estimator the surrogate is measured against:
log r4 = a + b log r3 fitted on the same training rates, ranked and given the
same exact budget.
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
    """An ensemble of device networks (trained one after another on the context's network, their
    parameters kept on the host) with the standardisation of its training set."""

    def __init__(self, ctx: Context, seed: int = 0, members: int = 1):
        self.ctx = ctx
        self.seed = seed
        self.members = int(members)
        self.params = []
        self.xm = self.xs = None
        self.ym = self.ys = None

    def fit(self, X, log_rate, epochs=400, batch=64, lr=2e-3):
        """Train every member on (X, log rate); returns the loss history of the first."""
        X = np.asarray(X, np.float64)
        y = np.asarray(log_rate, np.float64)
        self.xm, self.xs = X.mean(axis=0), X.std(axis=0) + 1e-12
        self.ym, self.ys = y.mean(), y.std() + 1e-12
        Xs, ys = (X - self.xm) / self.xs, (y - self.ym) / self.ys
        self.params, first = [], None
        for k in range(self.members):
            self.ctx.mlp_init(self.seed + 17 * k)
            h = self.ctx.mlp_train(Xs, ys, epochs=epochs, batch=min(batch, len(y)), lr=lr, seed=self.seed + 17 * k + 1)
            first = h if first is None else first
            self.params.append(self.ctx.mlp_params())
        return first

    def predict_all(self, X, bf16=True):
        """(members, n) predicted log rates."""
        X = np.asarray(X, np.float64)
        Xs = (X - self.xm) / self.xs
        out = []
        for p in self.params:
            self.ctx.mlp_set_params(p)
            out.append(self.ctx.mlp_predict(Xs, bf16=bf16).astype(np.float64) * self.ys + self.ym)
        return np.array(out)

    def predict(self, X, bf16=True):
        """Mean predicted log rate and the ensemble's spread (0 for one member)."""
        P = self.predict_all(X, bf16=bf16)
        return P.mean(axis=0), (P.std(axis=0) if len(P) > 1 else np.zeros(P.shape[1]))


class PowerLaw:
    """Network-free estimate log r4 = a + b log r3 (least squares on the training rates)."""

    def fit(self, rate3, rate4):
        m = (rate3 > 0) & (rate4 > 0)
        A = np.stack([np.ones(m.sum()), np.log(rate3[m])], axis=1)
        self.coef, *_ = np.linalg.lstsq(A, np.log(rate4[m]), rcond=None)
        return self

    def predict(self, rate3):
        r3 = np.where(rate3 > 0, rate3, np.nan)
        r4 = np.exp(self.coef[0] + self.coef[1] * np.log(r3))
        return np.where(np.isfinite(r4), r4, 0.0)


def kappa_weight(omega, nbe, grp_vel, mult):
    """Per-mode weight of a scattering-time change in kappa: mult * omega^2 n (n + 1) |v|^2."""
    v2 = np.sum(grp_vel * grp_vel, axis=2)
    return mult[:, None] * omega ** 2 * nbe * (nbe + 1.0) * v2


def mode_scores(rate3, rate4_pred, weight, spread=None, k_unc=1.0):
    """Predicted kappa change of each mode's four-phonon rate, weight * (1/r3 - 1/(r3 + r4)),
    scaled by 1 + k_unc * spread (the ensemble's spread of the log prediction)."""
    r3 = np.where(rate3 > 0, rate3, np.inf)
    d = weight * (1.0 / r3 - 1.0 / (r3 + np.maximum(rate4_pred, 0.0)))
    d = np.where(np.isfinite(d), d, 0.0)
    if spread is not None:
        d = d * (1.0 + k_unc * np.asarray(spread).reshape(d.shape))
    return d


def select_modes(scores, fraction):
    """Masks (n_q0,) of the top ceil(fraction * n_modes) modes by score (bit s = branch s)."""
    flat = np.asarray(scores).ravel()
    k = int(np.ceil(fraction * flat.size))
    top = np.argsort(-flat, kind="stable")[:k]
    sel = np.zeros(flat.size, bool)
    sel[top] = True
    sel = sel.reshape(scores.shape)
    masks = (sel.astype(np.int32) << np.arange(scores.shape[1])[None, :]).sum(axis=1).astype(np.int32)
    return masks, sel


def screened_rates4(ctx: Context, rate4_pred, masks, sigma=0.3767):
    """Four-phonon rates (nT, n_q0, Ndof): exact (one spring_linewidth4_modes call over every q0)
    for the selected branches, the prediction rate4_pred (nT, n_q0, Ndof) elsewhere."""
    exact = ctx.linewidth4_modes(1, masks, sigma=sigma)
    sel = ((masks[:, None] >> np.arange(rate4_pred.shape[-1])[None, :]) & 1).astype(bool)
    return np.where(sel[None], exact, rate4_pred), sel
