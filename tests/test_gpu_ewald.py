"""Device phonons with the dipole-dipole (Ewald) term against the oracle (LAPACK zheevd on the
short-range plus Ewald dynamical matrix, DynaMat_mod.f90:548-590): frequencies, occupations,
eigen-projectors and group velocities, Gamma (non-analytic term, finite-difference velocities)
included, on the grid and the irreducible set."""
import numpy as np
import pytest

from oracle import driver as D
from oracle import ewald as E
from oracle import phonons as P
from spring_b200 import synthetic as S
from spring_b200.api import from_crystal

pytestmark = pytest.mark.gpu


def _compare(ph, ref, n):
    np.testing.assert_allclose(np.sign(ph["omega"]) * ph["omega"] ** 2, np.sign(ref["omega"]) * ref["omega"] ** 2,
                               rtol=1e-10, atol=1e-9)
    np.testing.assert_allclose(ph["nbe"], ref["nbe"], rtol=1e-8, atol=1e-12)
    checked = 0
    for q in range(ref["omega"].shape[0]):
        w = ref["omega"][q]
        for s in range(n):
            gap = np.min(np.abs(np.delete(w, s) - w[s]))
            if gap < 1e-3 * max(1.0, abs(w[s])) or abs(w[s]) < 1e-3:
                continue
            e, f = ph["evec"][q, s], ref["evec"][q, s]
            np.testing.assert_allclose(np.outer(e, e.conj()), np.outer(f, f.conj()), atol=1e-9)
            np.testing.assert_allclose(ph["grp_vel"][q, s], ref["grp_vel"][q, s], rtol=1e-7, atol=1e-6)
            checked += 1
    assert checked > 0


@pytest.mark.parametrize("name,N,kw", [
    ("rocksalt2", 4, dict(rmesh=(5, 5, 5), decide=True, prec_ew=1e-8)),
    ("rocksalt2", 3, dict(rmesh=(4, 4, 4), decide=False, lmb=0.9, gmesh=(4, 5, 4))),   # even meshes
    ("rocksalt8", 2, dict(rmesh=(3, 3, 3), decide=True, prec_ew=1e-6)),
])
def test_phonons_with_dipole_term_match_oracle(name, N, kw):
    cr = S.make_polar(S.build(name))
    st = D.Setup(cr, (N, N, N), [300.0])
    ctx, info = from_crystal(cr, (N, N, N), st.temps, dipole=kw)
    ew = E.Ewald(cr.latvec, cr.G, cr.vol, cr.tau(), cr.eps, cr.zstar, **kw)
    lmb, gmesh, nr, ng = info["ewald"]
    assert abs(lmb - ew.lmb) < 1e-14 * ew.lmb and list(gmesh) == list(ew.gmesh)
    assert nr == len(ew.R) and ng == len(ew.Gp)
    args = (cr.latvec, cr.mass, cr.fc2_atm_num, cr.fc2_atm_indx, cr.fc2)
    for which, qs in ((0, st.q_pnt), (1, st.irr_q)):
        ref = P.get_phonon(*args, qs, st.temps, ewald=ew)
        _compare(ctx.get_phonons(which), ref, cr.ndof)
    ctx.close()


def test_dipole_term_off_restores_short_range_phonons():
    cr = S.make_polar(S.build("rocksalt2"))
    N = 4
    ctx, _ = from_crystal(cr, (N, N, N), [300.0], dipole=dict(rmesh=(5, 5, 5)))
    with_dd = ctx.get_phonons(0)["omega"].copy()
    ctx.set_dipole(None, None, None, None)
    ctx.compute_phonons([300.0])
    plain = ctx.get_phonons(0)["omega"]
    ctx.close()
    ref, _ = from_crystal(S.build("rocksalt2"), (N, N, N), [300.0])
    np.testing.assert_array_equal(plain, ref.get_phonons(0)["omega"])
    ref.close()
    assert np.abs(with_dd - plain).max() > 1.0   # the LO branch moves by rad/ps
