"""Surrogate-screened four-phonon kappa on the GPU: a network trained on exact rates of a coarse mesh
ranks the q0 blocks of a finer one; exact V4 on the top quarter plus the prediction elsewhere must land
far closer to the all-exact kappa than exact V4 on the same quarter without the network."""
import numpy as np
import pytest

from spring_b200 import surrogate as SG
from spring_b200 import synthetic as S
from spring_b200.api import from_crystal

pytestmark = pytest.mark.gpu

T = [300.0]
SIGMA = 0.3767


def _mesh(cr, N):
    ctx, info = from_crystal(cr, (N, N, N), T, with_fc4=True)
    ctx.reset_linewidths()
    lw3 = ctx.linewidth3(1, ctx.nq0, "gauss", SIGMA)[0][0]
    r4 = ctx.linewidth4(1, ctx.nq0, "gauss", SIGMA)[0]
    ph = ctx.get_phonons(1)
    q = ((cr.G / N) @ info["irr_q_pnt_int"].T.astype(float)).T
    X = SG.mode_features(ph["omega"], ph["grp_vel"], 2.0 * lw3, q)
    return ctx, info, lw3, r4, ph, X


def test_screened_kappa_beats_partial_exact():
    cr = S.build("rocksalt2", fc4=True)
    c8, _, _, r8, _, X8 = _mesh(cr, 8)
    y = r8.ravel()
    m = (y > 0) & (X8[:, 2] > 0)
    sur = SG.Surrogate(c8, seed=1)
    hist = sur.fit(X8[m], np.log(y[m]), epochs=600, batch=32, lr=2e-3)
    assert hist[-1] < 0.05 * hist[0]

    c10, info, lw3, r_exact, ph, X = _mesh(cr, 10)
    pred = np.exp(sur.predict(X, bf16=True)).reshape(c10.nq0, -1)
    ok = (r_exact.ravel() > 0) & (X[:, 2] > 0)
    assert np.median(np.abs(np.log(pred.ravel()[ok]) - np.log(r_exact.ravel()[ok]))) < 0.15

    w = SG.kappa_weight(ph["omega"], ph["nbe"][0], ph["grp_vel"], info["multiplicity"])
    order, _ = SG.rank_blocks(2.0 * lw3, pred, w)
    screened, exact_mask = SG.screened_rates4(c10, pred, order, 0.25, delta="gauss", sigma=SIGMA)
    assert exact_mask.sum() == int(np.ceil(0.25 * c10.nq0))
    np.testing.assert_allclose(screened[exact_mask], r_exact[exact_mask], rtol=1e-12)
    without = np.where(exact_mask[:, None], r_exact, 0.0)   # the same exact blocks, nothing elsewhere

    def kappa(r4):
        c10.set_linewidths((lw3 + 0.5 * r4)[None])
        k = c10.kappa_rta(info["Rxyz"])[0]
        return np.mean([k[0], k[4], k[8]])

    k_ex, k_scr, k_wo = kappa(r_exact), kappa(screened), kappa(without)
    err_scr, err_wo = abs(k_scr / k_ex - 1), abs(k_wo / k_ex - 1)
    assert err_scr < 5e-3, (k_ex, k_scr)
    assert err_scr < 0.25 * err_wo, (err_scr, err_wo)
    c8.close()
    c10.close()
