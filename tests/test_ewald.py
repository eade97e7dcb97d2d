"""The dipole-dipole (Ewald) term on the CPU: the oracle's restatement against known answers
(independence of the splitting parameter, the LO-TO splitting of a cubic diatomic crystal, the
acoustic sum rule at Gamma, the analytic q-derivative against finite differences), and the host
setup that the device library runs (src/Kappa/Src/EwaldParam.f90) against the oracle."""
import ctypes as ct

import numpy as np
import pytest

from oracle import ewald as E
from oracle import phonons as P
from spring_b200 import host_io as H
from spring_b200 import synthetic as S


@pytest.fixture(scope="module")
def polar():
    return S.make_polar(S.build("rocksalt2"))


def _ew(cr, **kw):
    kw.setdefault("rmesh", (7, 7, 7))
    return E.Ewald(cr.latvec, cr.G, cr.vol, cr.tau(), cr.eps, cr.zstar, **kw)


def test_splitting_parameter_independence(polar):
    """Real- plus reciprocal-space sums do not depend on Lmb once both have converged."""
    a = _ew(polar, decide=True, prec_ew=1e-10)
    b = _ew(polar, rmesh=(9, 9, 9), decide=False, lmb=1.3 * a.lmb, gmesh=[a.gmesh[0] + 4] * 3)
    q = polar.G @ np.array([0.1, 0.2, 0.3])
    Da, Db = a.dynmat(q, polar.mass), b.dynmat(q, polar.mass)
    assert np.abs(Da - Db).max() < 1e-8 * np.abs(Da).max()
    assert np.abs(Da - Da.conj().T).max() < 1e-14 * np.abs(Da).max()


def test_gradient_matches_finite_differences(polar):
    ew = _ew(polar, decide=True, prec_ew=1e-10)
    q = polar.G @ np.array([0.15, -0.2, 0.35])
    _, dD = ew.dynmat(q, polar.mass, grad=True)
    h = 1e-5
    for k in range(3):
        dq = np.zeros(3)
        dq[k] = h
        fd = (ew.dynmat(q + dq, polar.mass) - ew.dynmat(q - dq, polar.mass)) / (2 * h)
        assert np.abs(fd - dD[k]).max() < 1e-8 * np.abs(dD[k]).max()


def test_lo_to_splitting_and_acoustic_sum_rule():
    """Cubic diatomic crystal, isotropic spring model, Born charges +-Z, eps = e I: at Gamma the
    acoustic modes stay at zero (CSumq0) and the LO mode lies above the TO modes by
    4 pi e^2 Z^2 (1/m1 + 1/m2) / (V e) along every direction, the TO modes unchanged."""
    cr = S.rocksalt_primitive()
    S.make_fc2(cr, noise=0.0)
    S.make_polar(cr, z=1.986, eps=3.0)
    ew = _ew(cr, decide=True, prec_ew=1e-10)
    Dsr, _ = P.dynmat(cr.latvec, cr.mass, cr.fc2_atm_num, cr.fc2_atm_indx, cr.fc2, np.zeros(3))
    w0 = np.linalg.eigvalsh(Dsr + ew.dynmat(np.zeros(3), cr.mass))
    pred = 4 * np.pi * E.eV_A2 * 1.986 ** 2 * (1 / cr.mass[0] + 1 / cr.mass[1]) / (cr.vol * 3.0)
    for qhat in ([1.0, 0, 0], [1.0, 1.0, 0], [0.3, 0.5, 0.8], [1e-3, 0, 0]):
        w = np.linalg.eigvalsh(Dsr + ew.dynmat_na(np.array(qhat), cr.mass))
        assert np.abs(w[:3]).max() < 1e-12
        np.testing.assert_allclose(w[3:5], w0[3:5], rtol=1e-9)   # the sums converge to ~1e-10
        assert abs((w[5] - w0[5]) / pred - 1.0) < 1e-8


@pytest.mark.parametrize("decide", [True, False])
def test_host_setup_matches_oracle(polar, decide):
    """Lmb, Gmesh, the point counts, the constant part -Z(CConst) - CSumq0 and the Born-charge
    folded real-space terms of the C++ setup against the oracle's."""
    kw = dict(decide=True, prec_ew=1e-8, sup_cell=(5, 5, 5)) if decide else dict(decide=False, lmb=0.9, gmesh=(5, 7, 5))
    ew = _ew(polar, rmesh=(5, 5, 3), **kw)
    lib = H.load()
    nb = polar.nbasis
    lm = ct.c_double()
    gm = np.zeros(3, np.int32)
    cnt = np.zeros(2, np.int32)
    cc = np.zeros(2 * 9 * nb * nb)
    nr = 5 * 5 * 3
    hz = np.zeros(nr * 9 * nb * nb)
    f = lambda a, t: np.ascontiguousarray(a, t)
    rc = lib.spring_ewald_setup(H._ptr(f(polar.latvec.T, np.float64)), nb, H._ptr(f(polar.basis_frac, np.float64)),
                                H._ptr(f(polar.eps.T, np.float64)), H._ptr(f(polar.zstar.transpose(0, 2, 1), np.float64)),
                                int(decide), 1e-8, 0.9, H._ptr(f((5, 7, 5), np.int32)), H._ptr(f((5, 5, 3), np.int32)),
                                H._ptr(f((5, 5, 5), np.int32)), ct.byref(lm), H._ptr(gm), H._ptr(cnt), H._ptr(cc),
                                H._ptr(hz), hz.size)
    assert rc == 0, lib.spring_host_last_error()
    assert abs(lm.value - ew.lmb) < 1e-14 * ew.lmb
    assert list(gm) == list(ew.gmesh) and cnt[0] == nr and cnt[1] == int(np.prod(ew.gmesh))
    # oracle: -Z(CConst) - delta CSumq0, in (mu, nu, alpha, beta) order = Fortran C(beta, alpha, nu, mu)
    ref = -ew.combine(ew.cconst)
    for mu in range(nb):
        ref[mu, mu] -= ew.csum[mu]
    got = (cc[0::2] + 1j * cc[1::2]).reshape(nb, nb, 3, 3)
    np.testing.assert_allclose(got, ref, rtol=1e-11, atol=1e-13 * np.abs(ref).max())
    # real-space terms: sum_R e^{iqR} HZ_R equals Z(RealSpaceEW(q)) for any q
    q = polar.G @ np.array([0.2, -0.1, 0.4])
    ph = np.exp(1j * (ew.R @ q))
    got_r = (ph[:, None] * hz.reshape(nr, -1)).sum(axis=0).reshape(nb, nb, 3, 3)
    ref_r = ew.combine(ew.real_space(q))
    np.testing.assert_allclose(got_r, ref_r, rtol=1e-10, atol=1e-12 * np.abs(ref_r).max())


def test_host_setup_refuses_bad_input(polar):
    lib = H.load()
    f = lambda a, t: np.ascontiguousarray(a, t)
    bad_eps = np.diag([1.0, -1.0, 1.0])
    rc = lib.spring_ewald_setup(H._ptr(f(polar.latvec.T, np.float64)), 2, H._ptr(f(polar.basis_frac, np.float64)),
                                H._ptr(f(bad_eps, np.float64)), H._ptr(f(polar.zstar, np.float64)), 1, 1e-6, 0.8,
                                None, H._ptr(f((3, 3, 3), np.int32)), H._ptr(f((5, 5, 5), np.int32)),
                                None, None, None, None, None, 0)
    assert rc != 0 and b"determinant" in lib.spring_host_last_error()


def test_driver_reads_the_dipole_namelists(polar):
    """spring_kappa -dry-run with Force_dd: dielec, BornZ, Sup_Cell and &EwaldInfo reach the setup,
    whose Lmb and Gmesh equal the oracle's DecideEwaldParameters."""
    import json
    import os
    import subprocess
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        H.write_input(os.path.join(d, "input.nml"), polar, "MgO", (4, 4, 4),
                      dipole=dict(rmesh=(5, 5, 3), prec_ew=1e-8, sup_cell=(7, 7, 7)))
        for o in (2, 3):
            H.write_fc(os.path.join(d, H.fc_file_name(o, "MgO", 300.0)), o, getattr(polar, f"fc{o}_atm_num"),
                       getattr(polar, f"fc{o}_atm_indx"), getattr(polar, f"fc{o}"))
        r = subprocess.run([H.CLI, "-inp", "input.nml", "-T", "300", "-dry-run"], cwd=d, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        info = json.loads(r.stdout)
    ew = _ew(polar, rmesh=(5, 5, 3), decide=True, prec_ew=1e-8, sup_cell=(7, 7, 7))
    assert info["force_dd"] and abs(info["ewald_lmb"] - ew.lmb) < 1e-13 * ew.lmb
    assert info["ewald_gmesh"] == list(ew.gmesh) and info["ewald_points"] == [75, int(np.prod(ew.gmesh))]
