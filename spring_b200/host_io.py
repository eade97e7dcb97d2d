"""The reference's input and output files, through libspring_host.so (include/spring_host.h).

write_fc / read_fc: FC2nd_/FC3rd_/FC4th_<prefix><T>K_F.h5 in the layout r2ndFC / r3rdFC / r4thFC read
(src/Kappa/Src/hdf5_wrap_mod.f90:40-337).  read_f64: one dataset of an output file such as
kappa_<prefix><T>K.h5.  write_input: an input.nml with the namelists kappa.x reads.  The command-line
driver ``spring_b200/spring_kappa`` runs kappa.x's flow on these files (its arguments are kappa.x's).
Arrays follow the package's convention: C-order numpy arrays whose memory is the Fortran array.
"""
from __future__ import annotations

import ctypes as ct
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
HOST_LIB = os.path.join(_HERE, "libspring_host.so")
CLI = os.path.join(_HERE, "spring_kappa")
_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(HOST_LIB):
            raise ImportError(f"{HOST_LIB} is missing: build with `python -m spring_b200.build`")
        lib = ct.CDLL(HOST_LIB)
        P, I = ct.c_void_p, ct.c_int
        sig = {"spring_h5_write_fc": [ct.c_char_p, I, I, I, P, P, P],
               "spring_h5_fc_dims": [ct.c_char_p, I, P, P],
               "spring_h5_read_fc": [ct.c_char_p, I, I, I, P, P, P],
               "spring_h5_write_kappa": [ct.c_char_p, P, I, I, P, P, P, P],
               "spring_h5_read_f64": [ct.c_char_p, ct.c_char_p, P, P, P, ct.c_longlong],
               "spring_h5_write_restart": [ct.c_char_p, I, I, I, I, P],
               "spring_h5_read_restart": [ct.c_char_p, I, I, P, P],
               "spring_ewald_setup": [P, I, P, P, P, I, ct.c_double, ct.c_double, P, P, P, P, P, P, P, P,
                                      ct.c_longlong]}
        for name, args in sig.items():
            getattr(lib, name).argtypes = args
            getattr(lib, name).restype = I
        lib.spring_host_last_error.restype = ct.c_char_p
        _lib = lib
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ct.c_void_p)


def _check(rc):
    if rc != 0:
        raise OSError(load().spring_host_last_error().decode())


def fc_file_name(order: int, prefix: str, T: float) -> str:
    """'FC2nd_'//prefix//Temp_char//'K_F.h5' with Temp_char = F6.1 of T (main.f90:182-195)."""
    tag = {2: "FC2nd_", 3: "FC3rd_", 4: "FC4th_"}[order]
    return f"{tag}{prefix}{T:6.1f}".replace(" ", "") + "K_F.h5"


def write_fc(path, order, atm_num, atm_indx, fc):
    atm_num = np.ascontiguousarray(atm_num, np.int32)
    atm_indx = np.ascontiguousarray(atm_indx, np.int32)
    fc = np.ascontiguousarray(fc, np.float64)
    nb, na = atm_indx.shape[0], atm_indx.shape[1]
    _check(load().spring_h5_write_fc(os.fsencode(path), int(order), nb, na, _ptr(atm_num), _ptr(atm_indx), _ptr(fc)))


def read_fc(path, order):
    """(atm_num (Nb,), atm_indx (Nb, Na, 4), fc) with fc shaped like the synthetic crystal's."""
    lib = load()
    nb, na = ct.c_int(), ct.c_int()
    _check(lib.spring_h5_fc_dims(os.fsencode(path), int(order), ct.byref(nb), ct.byref(na)))
    nb, na = nb.value, na.value
    num = np.zeros(nb, np.int32)
    idx = np.zeros((nb, na, 4), np.int32)
    shape = {2: (nb, na, 3, 3, 1), 3: (nb, na, na, 3, 3, 3), 4: (nb, na, na, na, 3, 3, 3, 3)}[order]
    fc = np.zeros(shape)
    _check(lib.spring_h5_read_fc(os.fsencode(path), int(order), nb, na, _ptr(num), _ptr(idx), _ptr(fc)))
    return num, idx, fc


def read_f64(path, name):
    """A double dataset as a C-order array with the Fortran dimensions reversed."""
    lib = load()
    rank = ct.c_int()
    dims = (ct.c_longlong * 8)()
    _check(lib.spring_h5_read_f64(os.fsencode(path), name.encode(), ct.byref(rank), dims, None, 0))
    fd = [int(dims[i]) for i in range(rank.value)]
    out = np.zeros(int(np.prod(fd)) if fd else 1)
    _check(lib.spring_h5_read_f64(os.fsencode(path), name.encode(), ct.byref(rank), dims, _ptr(out), out.size))
    return out.reshape(fd[::-1])


def write_restart(path, progress, lw):
    """Restart file (w_RestartLW): progress (i0, complete) and LW_data, lw shaped (Nq0, Ndof)."""
    lw = np.ascontiguousarray(lw, np.float64)
    _check(load().spring_h5_write_restart(os.fsencode(path), lw.shape[1], lw.shape[0], int(progress[0]),
                                          int(progress[1]), _ptr(lw)))


def read_restart(path, ndof, nq0):
    prog = np.zeros(2, np.int32)
    lw = np.zeros((nq0, ndof))
    _check(load().spring_h5_read_restart(os.fsencode(path), int(ndof), int(nq0), _ptr(prog), _ptr(lw)))
    return (int(prog[0]), int(prog[1])), lw


def write_input(path, cr, prefix, qmesh, sigma=None, isotope=False, g2iso=None, four_phonon=False,
                selection3=("D", "D", "D"), time_rev=0, write_restart=False, read_restart=False, dipole=None,
                point_defect=None):
    """An input.nml with &FCInfo, &CrystalInfo, &AtmInfo (unit_mod.f90:64-209) and &AnhInfo
    (Helper_m.f90:37-132) for a synthetic crystal: one species per distinct mass.  ``dipole``
    (dict: rmesh, and optionally decide, prec_ew, lmb, gmesh, sup_cell) adds Force_dd, the crystal's
    dielec and BornZ, and &EwaldInfo (EwaldParam.f90).  ``point_defect`` (dict: def_pos, Mass_def,
    rho_def, qMesh_pd, NumDef_sup, cell_atom, MatInvFull, OptcTherm, IFC2_file_pd; any subset) writes
    &PointDefInfo (Helper_m.f90:135-307)."""
    masses, typ = [], []
    for m in cr.mass:
        if float(m) not in masses:
            masses.append(float(m))
        typ.append(masses.index(float(m)) + 1)
    L = []
    L.append("&FCInfo\n    prefix = '%s'\n    SecondFC = .true.\n    ThirdFC = .true.\n    FourthFC = %s\n"
             % (prefix, ".true." if four_phonon else ".false."))
    if dipole is not None:
        L.append("    Force_dd = .true.\n")
    L.append("/\n&CrystalInfo\n    Nbasis = %d\n    Ntyp = %d\n" % (cr.nbasis, len(masses)))
    if dipole is not None:
        L.append("    Sup_Cell = %d %d %d\n" % tuple(dipole.get("sup_cell", (5, 5, 5))))
    for k in range(3):
        L.append("    Latvec(:, %d) = %s\n" % (k + 1, " ".join("%.16g" % v for v in cr.latvec[:, k])))
    L.append("/\n&AtmInfo\n")
    for i in range(cr.nbasis):
        L.append("    atm_pos(:, %d) = %s\n" % (i + 1, " ".join("%.16g" % v for v in cr.basis_frac[i])))
    L.append("    typ_indx = %s\n" % " ".join(str(t) for t in typ))
    L.append("    mass = %s\n" % " ".join("%.10g" % m for m in masses))
    if dipole is not None:
        for j in range(3):
            L.append("    dielec(:, %d) = %s\n" % (j + 1, " ".join("%.16g" % cr.eps[i, j] for i in range(3))))
        for mu in range(cr.nbasis):
            for j in range(3):
                L.append("    BornZ(:, %d, %d) = %s\n" % (j + 1, mu + 1,
                                                         " ".join("%.16g" % cr.zstar[mu][i, j] for i in range(3))))
    L.append("/\n")
    if dipole is not None:
        L.append("&EwaldInfo\n    decide_EwParam = %s\n    prec_Ew = %.16g\n    Lmb = %.16g\n"
                 % (".true." if dipole.get("decide", True) else ".false.", dipole.get("prec_ew", 1e-6),
                    dipole.get("lmb", 0.8)))
        if dipole.get("gmesh") is not None:
            L.append("    Gmesh = %d %d %d\n" % tuple(dipole["gmesh"]))
        L.append("    Rmesh = %d %d %d\n/\n" % tuple(dipole["rmesh"]))
    if point_defect is not None:
        L.append("&PointDefInfo\n")
        for k, v in point_defect.items():
            if isinstance(v, bool):
                L.append("    %s = %s\n" % (k, ".true." if v else ".false."))
            elif isinstance(v, str):
                L.append("    %s = '%s'\n" % (k, v))
            elif k == "cell_atom":
                for j, col in enumerate(v):
                    L.append("    cell_atom(:, %d) = %s\n" % (j + 1, " ".join(str(int(x)) for x in col)))
            elif np.ndim(v) == 0:
                L.append("    %s = %.16g\n" % (k, v))
            else:
                L.append("    %s = %s\n" % (k, " ".join("%.16g" % x for x in np.ravel(v))))
        L.append("/\n")
    L.append("&AnhInfo\n    qmesh = %d %d %d\n    time_rev = %d\n" % (*qmesh, time_rev))
    L.append("    SelectionRule3 = %s\n" % " ".join("'%s'" % s for s in selection3))
    if sigma is not None:
        L.append("    Sigma = %.16g\n" % sigma)
    if isotope:
        L.append("    isotope = .true.\n    g2iso = %s\n" % " ".join("%.16g" % g for g in g2iso))
    if four_phonon:
        L.append("    FourPhonon = .true.\n")
    if write_restart:
        L.append("    WriteRestart = .true.\n")
    if read_restart:
        L.append("    ReadRestart = .true.\n")
    L.append("/\n")
    with open(path, "w") as f:
        f.write("".join(L))
