"""The reference's file formats on the CPU: FC files written in the layout r2ndFC / r3rdFC / r4thFC
read (src/Kappa/Src/hdf5_wrap_mod.f90:40-337) read back bit-exactly; the kappa result file's datasets;
the namelist reader and the command-line driver's input stage (-dry-run, no GPU)."""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

from spring_b200 import host_io as H
from spring_b200 import synthetic as S


@pytest.fixture(scope="module")
def cr4():
    return S.build("rocksalt2", fc4=True)


@pytest.mark.parametrize("order", [2, 3, 4])
def test_fc_file_round_trip(cr4, order):
    num, idx, fc = {2: (cr4.fc2_atm_num, cr4.fc2_atm_indx, cr4.fc2), 3: (cr4.fc3_atm_num, cr4.fc3_atm_indx, cr4.fc3),
                    4: (cr4.fc4_atm_num, cr4.fc4_atm_indx, cr4.fc4)}[order]
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, H.fc_file_name(order, "MgO", 300.0))
        H.write_fc(p, order, num, idx, fc)
        with open(p, "rb") as f:
            assert f.read(8) == b"\x89HDF\r\n\x1a\n"  # an HDF5 file (superblock version 0 follows)
        n2, i2, f2 = H.read_fc(p, order)
        assert np.array_equal(n2, num)
        assert np.array_equal(i2[:, : idx.shape[1]], idx)
        assert np.array_equal(f2.reshape(-1), np.ascontiguousarray(fc).reshape(-1))


def test_fc_file_names_follow_the_reference():
    assert H.fc_file_name(2, "MgO", 300.0) == "FC2nd_MgO300.0K_F.h5"
    assert H.fc_file_name(4, "X", 1200.0) == "FC4th_X1200.0K_F.h5"


def test_kappa_file_datasets():
    lib = H.load()
    rng = np.random.default_rng(0)
    nd, nq0 = 6, 10
    kap = rng.normal(size=9)
    lw = rng.normal(size=(nq0, 2 * nd))
    p3 = rng.normal(size=(nq0, 2 * nd))
    mk = rng.normal(size=(nd, 9))
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "kappa_X300.0K.h5")
        pd = rng.normal(size=(nq0, 2 * nd))
        assert lib.spring_h5_write_kappa(p.encode(), H._ptr(kap), nd, nq0, H._ptr(lw), H._ptr(p3), H._ptr(mk),
                                         H._ptr(pd)) == 0
        assert np.array_equal(H.read_f64(p, "ThermalConductivityTensor"), kap)
        assert np.array_equal(H.read_f64(p, "LineWidth"), lw)
        assert np.array_equal(H.read_f64(p, "PhaseSpace3rd"), p3)
        assert np.array_equal(H.read_f64(p, "ModeResolvedKappa"), mk)
        assert np.array_equal(H.read_f64(p, "Scatter_pd"), pd)
        with pytest.raises(OSError):
            H.read_f64(p, "NoSuchDataset")


def test_reader_refuses_non_hdf5():
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "x.h5")
        open(p, "wb").write(b"not an hdf5 file" * 64)
        with pytest.raises(OSError, match="not an HDF5 file"):
            H.read_fc(p, 2)


def test_driver_reads_namelists_and_fc_files(cr4):
    """spring_kappa -dry-run: the namelists (with array sections, repeat counts, comments and
    defaults) and the three FC files, as the driver will hand them to the library."""
    with tempfile.TemporaryDirectory() as d:
        H.write_input(os.path.join(d, "input.nml"), cr4, "MgO", (6, 6, 6), sigma=0.5, isotope=True,
                      g2iso=[1e-3, 1e-3], four_phonon=True, selection3=("D", "A", "O"))
        # a comment and a repeat count, as a user's file may have them
        with open(os.path.join(d, "input.nml"), "a") as f:
            f.write("! trailing comment\n&Other\n  x = 3*0.5 ! comment\n/\n")
        for order, (num, idx, fc) in {2: (cr4.fc2_atm_num, cr4.fc2_atm_indx, cr4.fc2),
                                      3: (cr4.fc3_atm_num, cr4.fc3_atm_indx, cr4.fc3),
                                      4: (cr4.fc4_atm_num, cr4.fc4_atm_indx, cr4.fc4)}.items():
            H.write_fc(os.path.join(d, H.fc_file_name(order, "MgO", 300.0)), order, num, idx, fc)
        r = subprocess.run([H.CLI, "-inp", "input.nml", "-T", "300", "-dry-run"], cwd=d, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        info = json.loads(r.stdout)
    assert info["prefix"] == "MgO" and info["T"] == "300.0" and info["nbasis"] == 2
    np.testing.assert_allclose(info["mass"], cr4.mass, rtol=1e-9)
    np.testing.assert_allclose(np.array(info["latvec"]).reshape(3, 3).T, cr4.latvec, rtol=1e-15)
    assert info["qmesh"] == [6, 6, 6] and info["shift"] == [0, 0, 0] and info["sigma"] == 0.5
    assert info["isotope"] and info["four_phonon"] and info["g2iso"] == [1e-3, 1e-3]
    assert info["pol3"] == [1, 6, 1, 3, 4, 6]      # PolarizationStrtEnd of D, A, O
    assert info["pol4"] == [1, 6] * 4              # default SelectionRule4
    assert info["na2"] == cr4.fc2_atm_indx.shape[1] and info["na3"] == 7 and info["na4"] == 7
    np.testing.assert_allclose(info["fc2_sum"], cr4.fc2.sum(), rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(info["fc3_sumsq"], (cr4.fc3 ** 2).sum(), rtol=1e-12)
    np.testing.assert_allclose(info["fc4_sumsq"], (cr4.fc4 ** 2).sum(), rtol=1e-12)
    assert info["n_rotations"] == 48               # O_h for the rocksalt primitive cell


def test_driver_reports_missing_files(cr4):
    with tempfile.TemporaryDirectory() as d:
        H.write_input(os.path.join(d, "input.nml"), cr4, "MgO", (4, 4, 4))
        r = subprocess.run([H.CLI, "-inp", "input.nml", "-T", "300", "-dry-run"], cwd=d, capture_output=True, text=True)
        assert r.returncode != 0 and "FC2nd_MgO300.0K_F.h5" in r.stderr


def test_restart_file_round_trip():
    lw = np.random.default_rng(1).normal(size=(29, 6))
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "MgO300.0K_LW_Restart.h5")
        H.write_restart(p, (17, 1), lw)
        prog, back = H.read_restart(p, 6, 29)
        assert prog == (17, 1)
        assert np.array_equal(back, lw)
        with pytest.raises(OSError, match="not \\(Ndof, Nq0\\)"):
            H.read_restart(p, 6, 30)  # another run's file
