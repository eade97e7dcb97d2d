"""Point-defect scattering in the oracle (src/Kappa/Src/point_defect_m.f90, GreensFunc_m.f90):
the tetrahedron vertex coefficients against their defining integrals, and the T-matrix rate's
optical-theorem and tetrahedron forms against each other in the Born limit."""
import numpy as np
import pytest

from oracle import driver as D
from spring_b200 import synthetic as S


def _c_and_d(E, W):
    Ws, v, cf = D.pd_coeff(E, W)
    return Ws, -cf.imag / np.pi, cf.real


@pytest.mark.parametrize("W", [[1.0, 2.5, 3.2, 5.0], [0.3, 0.9, 1.0, 4.0], [2.0, 2.1, 3.7, 3.9]])
def test_delta_weights_integrate_to_one(W):
    """sum_v c_v(E) is the tetrahedron's density of states: it integrates to 1 over E."""
    E = np.linspace(W[0] - 0.1, W[-1] + 0.1, 200001)
    tot = np.array([_c_and_d(e, W)[1].sum() for e in E[::50]])
    integral = np.trapezoid(tot, E[::50])
    assert abs(integral - 1.0) < 2e-4


@pytest.mark.parametrize("W", [
    [1.0, 2.5, 3.2, 5.0],          # all distinct
    [1.0, 1.0, 3.2, 5.0],          # one equal pair (1, 2)
    [1.0, 2.5, 2.5, 5.0],          # one equal pair (2, 3)
    [1.0, 1.0, 1.0, 5.0],          # vertices 1-3 equal
    [1.0, 4.0, 4.0, 4.0],          # vertices 2-4 equal
    [1.0, 1.0, 4.0, 4.0],          # two pairs
])
@pytest.mark.parametrize("E", [-2.0, 0.5, 6.0, 9.0])
def test_real_part_is_the_hilbert_transform_of_the_delta_weights(W, E):
    """Outside the tetrahedron's energy range d_v(E) = int c_v(E') / (E - E') dE' (Coeff = d - i pi c
    is the vertex weight of 1 / (E - E' + i0)); the degenerate forms are checked with tetrahedra
    whose energies are split by 1e-4 (about the same limit)."""
    Wt = np.array(W, float)
    split = Wt + np.array([0.0, 1e-4, 2e-4, 3e-4]) * (np.diff(np.r_[Wt, np.inf]) == 0).cumsum()  # a nearby distinct one
    Ep = np.linspace(Wt[0], Wt[-1], 400001)[1:-1]
    for Wq, tol in ((Wt, 2e-4), ):
        _, _, d = _c_and_d(E, Wq)
        cs = np.array([_c_and_d(e, split)[1] for e in Ep[::40]])
        ref = np.trapezoid(cs / (E - Ep[::40, None]), Ep[::40], axis=0)
        np.testing.assert_allclose(d, ref, rtol=tol * 10, atol=tol * np.abs(ref).max())


@pytest.fixture(scope="module")
def setup4():
    cr = S.build("rocksalt2")
    return cr, D.Setup(cr, (4, 4, 4), [300.0])


def test_perturbation_matrix(setup4):
    cr, _ = setup4
    num, idx, fc = S.defect_fc2(cr, site=0, scale=1.2)
    mdef = np.array([40.0, cr.mass[1]])
    vfc, vm = D.pd_perturbation(cr, num, idx, fc, mdef)
    V = vfc.reshape(6, 6).T          # V(row, col)
    wthz = np.sqrt(1.60217733 * 6.02214076 * 10.0) * 10.0
    onsite = cr.fc2[0, 0, :, :, 0]   # fC(1, beta, alpha, 1, 1) at [alpha][beta]
    np.testing.assert_allclose(V[:3, :3], 0.2 * onsite.T / cr.mass[0] * wthz ** 2, rtol=1e-12)
    assert np.abs(V[3:, :]).max() == 0 and np.abs(V[:, 3:]).max() == 0
    np.testing.assert_allclose(np.diag(vm.reshape(6, 6)), [(40.0 - cr.mass[0]) / cr.mass[0]] * 3 + [0.0] * 3)


def test_born_limit_optical_theorem_equals_tetrahedron_sum(setup4):
    """With T = V + V G V the optical theorem gives pi/NT sum c |e^H V e0|^2 and the tetrahedron form
    pi/NT sum c |e^H T e0|^2: equal to second order in V, so their relative difference shrinks in
    proportion to the perturbation."""
    cr, st = setup4
    diffs = []
    for eps in (1e-2, 1e-3):
        num, idx, fc = S.defect_fc2(cr, site=0, scale=1.0 + eps)
        mdef = np.array([cr.mass[0] * (1.0 + eps), cr.mass[1]])
        a = D.pd_rates(st, (4, 4, 4), num, idx, fc, mdef, 1e-3, mat_inv_full=False, optc_therm=True)
        b = D.pd_rates(st, (4, 4, 4), num, idx, fc, mdef, 1e-3, mat_inv_full=False, optc_therm=False)
        big = a > 1e-3 * a.max()
        diffs.append(np.abs(a[big] / b[big] - 1.0).max())
        assert np.all(a[0, :3] == 0) and np.all(b[0, :3] == 0)    # Gamma acoustic modes
    assert diffs[0] < 0.2 and diffs[1] < 0.15 * diffs[0]


def test_driver_reads_point_defect_namelist():
    """&PointDefInfo through spring_kappa -dry-run: defect masses mapped onto def_pos, the perturbed
    FC2 file read, the defaults of ReadPointDefVar, and its input checks."""
    import json
    import os
    import subprocess
    import tempfile
    from spring_b200 import host_io as H
    cr = S.build("rocksalt2")
    num, idx, fc = S.defect_fc2(cr, site=1, scale=1.1)
    with tempfile.TemporaryDirectory() as d:
        for o in (2, 3):
            H.write_fc(os.path.join(d, H.fc_file_name(o, "MgO", 300.0)), o, getattr(cr, f"fc{o}_atm_num"),
                       getattr(cr, f"fc{o}_atm_indx"), getattr(cr, f"fc{o}"))
        H.write_fc(os.path.join(d, "FC2nd_MgO300.0K_F_pd.h5"), 2, num, idx, fc)

        def run(pd):
            H.write_input(os.path.join(d, "input.nml"), cr, "MgO", (4, 4, 4), point_defect=pd)
            return subprocess.run([H.CLI, "-inp", "input.nml", "-T", "300", "-dry-run"], cwd=d, capture_output=True,
                                  text=True)
        r = run(dict(def_pos=[0, 1], Mass_def=[32.06], NumDef_sup=1, cell_atom=[[0, 0, 0, 2]], qMesh_pd=[5, 5, 5]))
        assert r.returncode == 0, r.stderr
        info = json.loads(r.stdout)
        assert info["point_defect"] and info["qmesh_pd"] == [5, 5, 5] and info["rho_def"] == 1e-6
        assert info["mat_inv_full"] and info["optc_therm"] and info["ifc2_file_pd"] == "FC2nd_MgO300.0K_F_pd.h5"
        np.testing.assert_allclose(info["mass_def"], [cr.mass[0], 32.06])
        assert run(dict(Mass_def=[32.06], NumDef_sup=1)).returncode != 0            # no def_pos
        assert run(dict(def_pos=[1, 1], Mass_def=[32.06], NumDef_sup=1, cell_atom=[[0, 0, 0, 1]])).returncode != 0
        assert run(dict(def_pos=[0, 1], Mass_def=[32.06])).returncode != 0          # NumDef_sup = 0
