"""Point-defect scattering rates on the GPU (spring_linewidth_pd) against the oracle's restatement
of ScatterRatePointDefect (src/Kappa/Src/point_defect_m.f90:139-376) with every combination of
MatInvFull and OptcTherm, and their 0.5 x rate contribution to LW_Allq0 (main.f90:685).

The rate depends on the eigenvector gauge inside degenerate levels of the defect mesh (the vertex
weights of a branch differ between degenerate branches, so sum_s w e e^H is not a projector sum),
as the reference's does on LAPACK's; the tests therefore give both sides the oracle's phonons."""
import numpy as np
import pytest

from oracle import driver as D
from oracle import phonons as P
from spring_b200 import synthetic as S
from spring_b200.api import from_crystal

pytestmark = pytest.mark.gpu


def _pd_phonons(cr, mesh):
    _, qf, _ = D.make_tetrahedron(mesh, cr.G, zero_centered=True)
    ph = P.get_phonon(cr.latvec, cr.mass, cr.fc2_atm_num, cr.fc2_atm_indx, cr.fc2, qf, [300.0])
    return dict(evec=ph["evec"], omega=ph["omega"])


@pytest.mark.parametrize("mat_inv_full,optc_therm", [(True, True), (True, False), (False, True), (False, False)])
def test_point_defect_rates_match_oracle(mat_inv_full, optc_therm):
    cr = S.build("rocksalt2")
    N, Npd = 4, (5, 5, 5)
    st = D.Setup(cr, (N, N, N), [300.0])
    num, idx, fc = S.defect_fc2(cr, site=0, scale=1.2)
    mdef = np.array([40.078, cr.mass[1]])     # Ca on the Mg site
    ctx, _ = from_crystal(cr, (N, N, N), st.temps, phonons={"grid": st.ph, "irr": st.ph0})
    ctx.set_point_defect(Npd, num, idx, fc, mdef, rho_def=1e-3, mat_inv_full=mat_inv_full, optc_therm=optc_therm,
                         phonons=_pd_phonons(cr, Npd))
    got = ctx.linewidth_pd()
    ref = D.pd_rates(st, Npd, num, idx, fc, mdef, 1e-3, mat_inv_full=mat_inv_full, optc_therm=optc_therm)
    assert np.abs(ref).max() > 0
    # the real parts of the vertex weights cancel catastrophically where vertex energies nearly
    # coincide (just above the 5e-5 degeneracy threshold), in the reference's formulas as here, so
    # last-bit differences of log() grow to ~1e-7; the delta-weight part alone agrees to 1e-10
    tol = 1e-10 if (not mat_inv_full and optc_therm) else 2e-6
    np.testing.assert_allclose(got, ref, rtol=tol, atol=1e-3 * tol * np.abs(ref).max())
    # the linewidth contribution
    ctx.reset_linewidths()
    ctx.linewidth_pd(add=True)
    np.testing.assert_allclose(ctx.get_linewidths()[0], 0.5 * got, rtol=1e-14, atol=0)
    ctx.close()


def test_point_defect_8_atom_cell():
    """Ndof 24: the large-cell branches of the Green's-function and T-matrix kernels.  The cubic
    cell's vertex energies are degenerate or nearly so at many tetrahedra, where the real-part
    weights are ill-conditioned; the optical theorem with T = V + V G V depends only on the delta
    weights, which are not, and is compared tightly."""
    cr = S.build("rocksalt8")
    st = D.Setup(cr, (2, 2, 2), [300.0])
    num, idx, fc = S.defect_fc2(cr, site=0, scale=1.1)
    mdef = cr.mass.copy()
    mdef[0] = 40.078
    ctx, _ = from_crystal(cr, (2, 2, 2), st.temps, phonons={"grid": st.ph, "irr": st.ph0})
    ctx.set_point_defect((3, 3, 3), num, idx, fc, mdef, rho_def=1e-3, mat_inv_full=False, optc_therm=True,
                         phonons=_pd_phonons(cr, (3, 3, 3)))
    got = ctx.linewidth_pd()
    ctx.close()
    ref = D.pd_rates(st, (3, 3, 3), num, idx, fc, mdef, 1e-3, mat_inv_full=False, optc_therm=True)
    np.testing.assert_allclose(got, ref, rtol=1e-8, atol=1e-10 * np.abs(ref).max())
