"""Surrogate-screened four-phonon kappa on the GPU: a network ensemble trained on exact rates of a
coarse mesh ranks the (q0, branch) blocks of a finer one; exact V4 on the top quarter of the blocks
plus the prediction elsewhere must land close to the all-exact kappa, and closer than a network-free
estimate (log r4 = a + b log r3 fitted on the same training rates) given the same exact budget."""
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
    ctx.set_precision("bf16x3")
    ctx.reset_linewidths()
    lw3 = ctx.linewidth3(1, ctx.nq0, "gauss", SIGMA)[0][0]
    r4 = ctx.linewidth4(1, ctx.nq0, "gauss", SIGMA)[0]
    ph = ctx.get_phonons(1)
    q = ((cr.G / N) @ info["irr_q_pnt_int"].T.astype(float)).T
    X = SG.mode_features(ph["omega"], ph["grp_vel"], 2.0 * lw3, q)
    return ctx, info, lw3, r4, ph, X


def test_screened_kappa_beats_network_free_estimate():
    cr = S.build("rocksalt2", fc4=True)
    c8, _, lw8, r8, _, X8 = _mesh(cr, 8)
    y = r8.ravel()
    m = (y > 0) & (X8[:, 2] > 0)
    sur = SG.Surrogate(c8, seed=1, members=3)
    hist = sur.fit(X8[m], np.log(y[m]), epochs=600, batch=32, lr=2e-3)
    assert hist[-1] < 0.05 * hist[0]
    pl = SG.PowerLaw().fit(X8[:, 2], y)

    c10, info, lw3, r_exact, ph, X = _mesh(cr, 10)
    mu, spread = sur.predict(X, bf16=True)
    pred = np.exp(mu).reshape(c10.nq0, -1)
    ok = (r_exact.ravel() > 0) & (X[:, 2] > 0)
    assert np.median(np.abs(mu[ok] - np.log(r_exact.ravel()[ok]))) < 0.15
    pred_pl = pl.predict(2.0 * lw3)

    w = SG.kappa_weight(ph["omega"], ph["nbe"][0], ph["grp_vel"], info["multiplicity"])

    def kappa(r4):
        c10.set_linewidths((lw3 + 0.5 * r4)[None])
        k = c10.kappa_rta(info["Rxyz"])[0]
        return np.mean([k[0], k[4], k[8]])

    def screened(p, unc):
        masks, sel = SG.select_modes(SG.mode_scores(2.0 * lw3, p, w, unc), 0.25)
        r, sel2 = SG.screened_rates4(c10, p[None], masks, sigma=SIGMA)
        assert np.array_equal(sel, sel2)
        np.testing.assert_allclose(r[0][sel], r_exact[sel], rtol=1e-9)
        return kappa(r[0])

    k_ex = kappa(r_exact)
    err_net = abs(screened(pred, spread) / k_ex - 1)
    err_pl = abs(screened(pred_pl, None) / k_ex - 1)
    assert err_net < 5e-3, (err_net, err_pl)
    assert err_net < err_pl, (err_net, err_pl)
    c8.close()
    c10.close()
