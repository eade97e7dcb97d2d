"""spring_kappa end to end on the GPU: kappa.x's command line, namelists and FC files in, the kappa
HDF5 file and the linewidth text file out, against the same computation through the Python API."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from spring_b200 import host_io as H
from spring_b200 import synthetic as S
from spring_b200.api import from_crystal

pytestmark = pytest.mark.gpu


def _run(cr, d, extra, **nml):
    H.write_input(os.path.join(d, "input.nml"), cr, "MgO", nml.pop("qmesh"), **nml)
    for order in (2, 3, 4):
        a = getattr(cr, f"fc{order}")
        if a is None:
            continue
        H.write_fc(os.path.join(d, H.fc_file_name(order, "MgO", 300.0)), order, getattr(cr, f"fc{order}_atm_num"),
                   getattr(cr, f"fc{order}_atm_indx"), a)
    r = subprocess.run([H.CLI, "-inp", "input.nml", "-T", "300", *extra], cwd=d, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    kap = H.read_f64(os.path.join(d, "kappa_MgO300.0K.h5"), "ThermalConductivityTensor")
    lwf = H.read_f64(os.path.join(d, "kappa_MgO300.0K.h5"), "LineWidth")
    txt = np.loadtxt(os.path.join(d, "linewidth_IBZ_MgO300.0K.txt"), comments="#")
    return kap, lwf, txt


def test_cli_three_phonon_tetrahedron_matches_api():
    cr = S.build("rocksalt2")
    N = 6
    with tempfile.TemporaryDirectory() as d:
        kap, lwf, txt = _run(cr, d, ["-Mode_resolved_k", "T"], qmesh=(N, N, N))
        mk = H.read_f64(os.path.join(d, "kappa_MgO300.0K.h5"), "ModeResolvedKappa")
    ctx, info = from_crystal(cr, (N, N, N), [300.0])
    ctx.reset_linewidths()
    ctx.linewidth3(1, ctx.nq0, delta="tetra", want=False)
    lw = ctx.get_linewidths()[0]
    om = ctx.get_phonons(1)["omega"]
    k_api, mk_api = ctx.kappa_rta(info["Rxyz"], mode=True)
    ctx.close()
    np.testing.assert_allclose(kap, k_api[0], rtol=1e-9, atol=1e-12 * np.abs(k_api).max())
    np.testing.assert_allclose(mk, mk_api[0], rtol=1e-9, atol=1e-12 * np.abs(mk_api).max())
    np.testing.assert_allclose(lwf[:, 6:], lw, rtol=1e-12, atol=0)
    np.testing.assert_allclose(lwf[:, :6], om, rtol=1e-12, atol=0)
    # the text file: Ndof frequencies then Ndof linewidths per irreducible point, 12 significant digits
    np.testing.assert_allclose(txt[:, :6], om, rtol=1e-11, atol=1e-11)
    np.testing.assert_allclose(txt[:, 6:], lw, rtol=1e-11, atol=1e-14)


def test_cli_four_phonon_isotope_gauss_bf16x3_matches_api():
    cr = S.build("rocksalt2", fc4=True)
    N = 4
    g2 = [1e-3, 1e-3]
    with tempfile.TemporaryDirectory() as d:
        kap, lwf, _ = _run(cr, d, ["-delta", "gauss", "-precision", "bf16x3"], qmesh=(N, N, N), sigma=0.8,
                           isotope=True, g2iso=g2, four_phonon=True)
    ctx, info = from_crystal(cr, (N, N, N), [300.0], with_fc4=True)
    ctx.set_precision("bf16x3")
    ctx.reset_linewidths()
    ctx.linewidth3(1, ctx.nq0, delta="gauss", sigma=0.8, want=False)
    ctx.linewidth_iso(1, ctx.nq0, g2, delta="gauss", sigma=0.8, want=False)
    ctx.linewidth4(1, ctx.nq0, delta="gauss", sigma=0.8, want=False)
    lw = ctx.get_linewidths()[0]
    k_api = ctx.kappa_rta(info["Rxyz"])[0]
    ctx.close()
    np.testing.assert_allclose(lwf[:, 6:], lw, rtol=1e-10, atol=1e-14)
    np.testing.assert_allclose(kap, k_api, rtol=1e-9, atol=1e-12 * np.abs(k_api).max())


def test_cli_restart_skips_the_points_already_done():
    """WriteRestart leaves the linewidth restart file; a run with ReadRestart from a file that holds
    only the first points (progress (k, 1)) computes the rest and gives the same results."""
    cr = S.build("rocksalt2")
    N = 5
    with tempfile.TemporaryDirectory() as d:
        kap1, lwf1, _ = _run(cr, d, [], qmesh=(N, N, N), write_restart=True)
        rfile = os.path.join(d, "Restart_MgO", "MgO300.0K_LW_Restart.h5")
        prog, lw = H.read_restart(rfile, 6, lwf1.shape[0])
        assert prog == (lwf1.shape[0], 1)
        np.testing.assert_array_equal(lw, lwf1[:, 6:])
        k = lwf1.shape[0] // 2
        part = lw.copy()
        part[k:] = 0.0
        H.write_restart(rfile, (k, 1), part)
        kap2, lwf2, _ = _run(cr, d, [], qmesh=(N, N, N), read_restart=True)
    np.testing.assert_allclose(lwf2, lwf1, rtol=1e-12, atol=0)
    np.testing.assert_allclose(kap2, kap1, rtol=1e-12, atol=1e-14 * np.abs(kap1).max())


def test_cli_dipole_term_matches_api():
    """Force_dd with &EwaldInfo through the driver: the same phonons, linewidths and kappa as the
    API with spring_set_dipole."""
    cr = S.make_polar(S.build("rocksalt2"))
    N = 4
    dip = dict(rmesh=(5, 5, 5), prec_ew=1e-8)
    with tempfile.TemporaryDirectory() as d:
        kap, lwf, _ = _run(cr, d, [], qmesh=(N, N, N), dipole=dip)
    ctx, info = from_crystal(cr, (N, N, N), [300.0], dipole=dip)
    ctx.reset_linewidths()
    ctx.linewidth3(1, ctx.nq0, delta="tetra", want=False)
    lw = ctx.get_linewidths()[0]
    om = ctx.get_phonons(1)["omega"]
    k_api = ctx.kappa_rta(info["Rxyz"])[0]
    ctx.close()
    np.testing.assert_allclose(lwf[:, :6], om, rtol=1e-12, atol=0)
    np.testing.assert_allclose(lwf[:, 6:], lw, rtol=1e-12, atol=0)
    np.testing.assert_allclose(kap, k_api, rtol=1e-9, atol=1e-12 * np.abs(k_api).max())


def test_cli_point_defect_matches_api():
    """&PointDefInfo through the driver: Scatter_pd, the ScatterRate_pd text file and the linewidths
    (0.5 x rate added) equal the API's spring_linewidth_pd on the same inputs."""
    cr = S.build("rocksalt2")
    N = 4
    num, idx, fc = S.defect_fc2(cr, site=0, scale=1.2)
    mdef = np.array([40.078, cr.mass[1]])
    pd = dict(def_pos=[1, 0], Mass_def=[40.078], NumDef_sup=1, cell_atom=[[0, 0, 0, 1]], qMesh_pd=[5, 5, 5],
              rho_def=1e-3)
    with tempfile.TemporaryDirectory() as d:
        H.write_fc(os.path.join(d, "FC2nd_MgO300.0K_F_pd.h5"), 2, num, idx, fc)
        kap, lwf, _ = _run(cr, d, [], qmesh=(N, N, N), point_defect=pd)
        spd = H.read_f64(os.path.join(d, "kappa_MgO300.0K.h5"), "Scatter_pd")
        txt = np.loadtxt(os.path.join(d, "ScatterRate_pd_IBZ_MgO300.0K.txt"), comments="#")
    ctx, info = from_crystal(cr, (N, N, N), [300.0])
    ctx.set_point_defect((5, 5, 5), num, idx, fc, mdef, rho_def=1e-3)
    ctx.reset_linewidths()
    ctx.linewidth3(1, ctx.nq0, delta="tetra", want=False)
    rate = ctx.linewidth_pd(add=True)
    lw = ctx.get_linewidths()[0]
    k_api = ctx.kappa_rta(info["Rxyz"])[0]
    ctx.close()
    np.testing.assert_allclose(spd[:, 6:], rate, rtol=1e-12, atol=0)
    np.testing.assert_allclose(txt[:, 6:], rate, rtol=1e-11, atol=1e-14)
    np.testing.assert_allclose(lwf[:, 6:], lw, rtol=1e-12, atol=0)
    np.testing.assert_allclose(kap, k_api, rtol=1e-9, atol=1e-12 * np.abs(k_api).max())
