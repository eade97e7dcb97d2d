"""Oracle driver — TEST INFRASTRUCTURE ONLY.

ctypes wrapper around ``oracle/_build/liboracle.so`` (the C++ FP64
restatement) plus the orchestration of ``kappa.x``'s driver loop
(``src/Kappa/Src/main.f90:552-766``) on top of it.  Used by tests/, by the
CPU-baseline leg of bench.py and by ``__graft_entry__.smoke`` as the checker;
the product never imports it.

Parity status: unpinned against reference outputs (the reference Fortran
cannot be built here and ships no golden vectors for this path); pinned by the
reference's in-code invariants and the known-answer tests in tests/.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np

from . import constants as C
from . import phonons as P

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
c128p = np.ctypeslib.ndpointer(dtype=np.complex128, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile the oracle (``make -C oracle``) and return the library path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "_build", "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "_build", "liboracle.so")
        if not os.path.exists(path):
            path = build()
        L = ct.CDLL(path)
        L.orc_make_tetrahedron.argtypes = [i32p, i32p, f64p, ct.c_int, i32p, f64p, i32p]
        L.orc_make_tetrahedron.restype = ct.c_int
        L.orc_irr_q.argtypes = [i32p, ct.c_int, i32p, ct.c_int, i32p, i32p, i32p, i32p, i32p]
        L.orc_irr_q.restype = ct.c_int
        L.orc_momentum3.argtypes = [i32p, i32p, i32p, i32p, i32p, i32p]
        L.orc_momentum3.restype = None
        L.orc_momentum4.argtypes = [i32p, i32p, i32p, i32p, i32p, ct.c_longlong, i64p]
        L.orc_momentum4.restype = ct.c_int
        L.orc_scatter_w3.argtypes = [ct.c_int, ct.c_int, i32p, i32p, f64p, f64p, f64p, ct.c_int, f64p, i32p,
                                     i32p, c128p, f64p, c128p, f64p, ct.c_int, i32p, f64p]
        L.orc_scatter_w3.restype = None
        L.orc_find_g_iver.argtypes = [ct.c_double, f64p, f64p, ct.c_int, f64p, f64p, f64p, f64p, i32p]
        L.orc_find_g_iver.restype = ct.c_int
        L.orc_lw3_tetra.argtypes = [ct.c_int, ct.c_int, f64p, f64p, f64p, f64p, i32p, i32p, i32p, f64p, f64p, f64p]
        L.orc_lw3_tetra.restype = None
        L.orc_lw3_gauss.argtypes = [ct.c_int, ct.c_int, f64p, f64p, f64p, f64p, i32p, i32p, i32p, ct.c_double,
                                    f64p, f64p]
        L.orc_lw3_gauss.restype = None
        L.orc_iso_w.argtypes = [ct.c_int, ct.c_int, c128p, f64p, c128p, f64p, f64p]
        L.orc_iso_w.restype = None
        L.orc_iso_lw_tetra.argtypes = [ct.c_int, ct.c_int, f64p, f64p, f64p, i32p, f64p]
        L.orc_iso_lw_tetra.restype = None
        L.orc_iso_lw_gauss.argtypes = [ct.c_int, ct.c_int, f64p, f64p, f64p, ct.c_double, f64p]
        L.orc_iso_lw_gauss.restype = None
        L.orc_velkron_symm.argtypes = [ct.c_int, ct.c_int, f64p, ct.c_int, f64p, i32p, f64p]
        L.orc_velkron_symm.restype = None
        L.orc_kappa_symm.argtypes = [ct.c_int, ct.c_int, ct.c_int, i32p, f64p, f64p, f64p, f64p, ct.c_int,
                                     ct.c_int, ct.c_double, ct.c_double, ct.c_double, f64p, ct.c_void_p]
        L.orc_kappa_symm.restype = None
        L.orc_kappa_full.argtypes = [ct.c_int, ct.c_int, i32p, i32p, f64p, f64p, f64p, f64p, ct.c_int, ct.c_int,
                                     ct.c_double, ct.c_double, ct.c_double, f64p]
        L.orc_kappa_full.restype = None
        L.orc_bte_iter.argtypes = [ct.c_int, ct.c_int, i32p, ct.c_int, i32p, i32p, i32p, i32p, i32p, f64p, f64p,
                                   f64p, f64p, i32p, ct.c_double, ct.c_double, ct.c_double, ct.c_int, f64p, f64p,
                                   f64p, f64p]
        L.orc_bte_iter.restype = ct.c_int
        L.orc_bte_iter_gauss.argtypes = [ct.c_int, ct.c_int, ct.c_double, ct.c_int, i32p, i32p, i32p, i32p, i32p,
                                         f64p, f64p, f64p, f64p, i32p, ct.c_double, ct.c_double, ct.c_double,
                                         ct.c_int, f64p, f64p, f64p, f64p]
        L.orc_bte_iter_gauss.restype = ct.c_int
        L.orc_num_threads.restype = ct.c_int
        _LIB = L
    return _LIB


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _c(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


# ----------------------------------------------------------------------------- mesh
def make_tetrahedron(mesh, G, shift=(0, 0, 0), zero_centered=True):
    mesh = _i(mesh)
    nq = int(np.prod(mesh))
    qi = np.zeros((nq, 3), np.int32)
    qf = np.zeros((nq, 3), np.float64)
    tet = np.zeros((6 * nq, 4), np.int32)
    rc = lib().orc_make_tetrahedron(mesh, _i(shift), _f(np.asarray(G).T), int(zero_centered), qi, qf, tet)
    if rc != 0:
        raise ValueError("make_tetrahedron: vertex outside the grid")
    return qi, qf, tet


def irr_q(mesh, W, q_pnt_int, time_rev=0):
    mesh = _i(mesh)
    nq = int(np.prod(mesh))
    mp = np.zeros(nq, np.int32)
    irr = np.zeros((nq, 3), np.int32)
    pos = np.zeros(nq, np.int32)
    mult = np.zeros(nq, np.int32)
    n = lib().orc_irr_q(mesh, len(W), _i(W), int(time_rev), _i(q_pnt_int), mp, irr, pos, mult)
    return dict(map=mp, irr_q_pnt_int=irr[:n].copy(), pos=pos, multiplicity=mult[:n].copy())


# ----------------------------------------------------------------------------- enumeration
def momentum3(mesh, q_pnt_int, q0_int):
    nq = int(np.prod(mesh))
    A = np.zeros((nq, 4), np.int32)
    Pm = np.zeros((nq, 2), np.int32)
    cnt = np.zeros(2, np.int32)
    lib().orc_momentum3(_i(mesh), _i(q_pnt_int), _i(q0_int), A, Pm, cnt)
    return A, Pm[: cnt[0]].copy(), (int(cnt[0]), int(cnt[1]))


def momentum4(mesh, q_pnt_int, q0_int, cap=None):
    nq = int(np.prod(mesh))
    if cap is None:
        cap = nq * nq
    A = np.zeros((nq, nq, 3), np.int32)
    Pm = np.zeros((cap, 3), np.int32)
    cnt = np.zeros(2, np.int64)
    rc = lib().orc_momentum4(_i(mesh), _i(q_pnt_int), _i(q0_int), A, Pm, int(cap), cnt)
    if rc != 0:
        raise ValueError("momentum4: capacity exceeded")
    return A, Pm[: cnt[0]].copy(), (int(cnt[0]), int(cnt[1]))


# ----------------------------------------------------------------------------- V3 / W
def fc3_derived(cr):
    """basisTyp(Na3,Nb) and atmPosR(3,Na3,Nb) of ``set_FC3`` (``src/Kappa/Src/FC3_mod.f90:49-94``)."""
    idx = cr.fc3_atm_indx
    btyp = _i(idx[:, :, 3])
    pos = np.einsum("ij,mnj->mni", cr.latvec, idx[:, :, :3].astype(np.float64))
    return btyp, _f(pos)


def scatter_w3(cr, q_pnt, q_pnt_int, q0_int, evec0, oneby0, evec, oneby, q1q2_perm):
    nb = cr.nbasis
    ndof = 3 * nb
    nq = q_pnt.shape[0]
    btyp, posr = fc3_derived(cr)
    out = np.zeros((nq, ndof, ndof, ndof), np.float64)
    lib().orc_scatter_w3(nb, cr.fc3.shape[1], _i(cr.fc3_atm_num), btyp, posr, _f(cr.fc3),
                         _f(1.0 / np.sqrt(cr.mass)), nq, _f(q_pnt), _i(q_pnt_int), _i(q0_int), _c(evec0),
                         _f(oneby0), _c(evec), _f(oneby), len(q1q2_perm), _i(q1q2_perm), out)
    return out   # [q1][s0][s1][s2] == Fortran Sctrq1(s2,s1,s0,q1)


def find_g_iver(Mqs, M, F, strict=False):
    g = np.zeros(1)
    I = np.zeros(4)
    Ms = np.zeros(4)
    Fs = np.zeros(4)
    perm = np.zeros(4, np.int32)
    e = lib().orc_find_g_iver(float(Mqs), _f(M), _f(F), int(strict), g, I, Ms, Fs, perm)
    return bool(e), float(g[0]), I, Ms, Fs, perm


def lw3_tetra(omega0, omega, nbe, sctr, tetra, Allq1q2, pol=None):
    ndof = omega.shape[1]
    nq = omega.shape[0]
    if pol is None:
        pol = np.array([[1, ndof]] * 3, np.int32)
    lw = np.zeros(ndof)
    p3q = np.zeros(ndof)
    p3 = np.zeros(1)
    lib().orc_lw3_tetra(ndof, nq, _f(omega0), _f(omega), _f(nbe), _f(sctr), _i(tetra), _i(Allq1q2), _i(pol),
                        lw, p3q, p3)
    return lw, p3q, float(p3[0])


def lw3_gauss(omega0, omega, nbe, sctr, Allq1q2, q_pnt_int, sigma, pol=None):
    ndof = omega.shape[1]
    nq = omega.shape[0]
    if pol is None:
        pol = np.array([[1, ndof]] * 3, np.int32)
    lw = np.zeros(ndof)
    p3q = np.zeros(ndof)
    lib().orc_lw3_gauss(ndof, nq, _f(omega0), _f(omega), _f(nbe), _f(sctr), _i(Allq1q2), _i(q_pnt_int),
                        _i(pol), float(sigma), lw, p3q)
    return lw, p3q


def iso_w(nb, evec0, omega0, evec, g2):
    nq = evec.shape[0]
    ndof = 3 * nb
    out = np.zeros((nq, ndof, ndof))
    lib().orc_iso_w(nb, nq, _c(evec0), _f(omega0), _c(evec), _f(g2), out)
    return out    # [q1][s0][s1] == Fortran W_iso(s1,s0,q1)


def iso_lw_tetra(omega0, omega, w_iso, tetra):
    ndof = omega.shape[1]
    lw = np.zeros(ndof)
    lib().orc_iso_lw_tetra(ndof, omega.shape[0], _f(omega0), _f(omega), _f(w_iso), _i(tetra), lw)
    return lw


def iso_lw_gauss(omega0, omega, w_iso, sigma):
    ndof = omega.shape[1]
    lw = np.zeros(ndof)
    lib().orc_iso_lw_gauss(ndof, omega.shape[0], _f(omega0), _f(omega), _f(w_iso), float(sigma), lw)
    return lw


# ----------------------------------------------------------------------------- kappa
def velkron_symm(grp_vel0, Rxyz, mult):
    nq0, ndof = grp_vel0.shape[:2]
    out = np.zeros((nq0, ndof, 9))
    # Rxyz(3,3,Nsym) column-major == C array [ns][col][row]
    R = _f(np.transpose(np.asarray(Rxyz), (0, 2, 1)))
    lib().orc_velkron_symm(ndof, nq0, _f(grp_vel0), len(Rxyz), R, _i(mult), out)
    return out


def kappa_symm(nq, irr_int, omega0, nbe0, lw, krn, vol, T, s_first=1, s_last=None, mode=False):
    nq0, ndof = omega0.shape
    if s_last is None:
        s_last = ndof
    kap = np.zeros(9)
    mk = np.zeros((ndof, 9)) if mode else None
    lib().orc_kappa_symm(ndof, nq, nq0, _i(irr_int), _f(omega0), _f(nbe0), _f(lw), _f(krn), s_first, s_last,
                         vol, T, C.kW_m_k, kap, mk.ctypes.data if mode else None)
    return (kap, mk) if mode else kap


def kappa_full(q_pnt_int, pos, omega, nbe, grp_vel, lw, vol, T, s_first=1, s_last=None):
    nq, ndof = omega.shape
    if s_last is None:
        s_last = ndof
    kap = np.zeros(9)
    lib().orc_kappa_full(ndof, nq, _i(q_pnt_int), _i(pos), _f(omega), _f(nbe), _f(grp_vel), _f(lw), s_first,
                         s_last, vol, T, C.kW_m_k, kap)
    return kap


# ----------------------------------------------------------------------------- pipeline
class Setup:
    """Mesh, irreducible set and phonons for one crystal / mesh / temperature list."""

    def __init__(self, cr, mesh, temps, W=None, Rxyz=None):
        from spring_b200 import synthetic as S
        self.cr = cr
        self.mesh = np.array(mesh, np.int32)
        self.temps = np.atleast_1d(np.asarray(temps, np.float64))
        self.nq = int(np.prod(self.mesh))
        self.q_pnt_int, self.q_pnt, self.tetra = make_tetrahedron(self.mesh, cr.G)
        if W is None:
            W, Rxyz = S.point_group(cr)
        self.W, self.Rxyz = W, Rxyz
        ir = irr_q(self.mesh, W, self.q_pnt_int)
        self.irr_int = ir["irr_q_pnt_int"]
        self.pos = ir["pos"]
        self.mult = ir["multiplicity"]
        self.nq0 = self.irr_int.shape[0]
        Ru = cr.G / self.mesh[None, :]
        self.irr_q = (Ru @ self.irr_int.T.astype(np.float64)).T
        args = (cr.latvec, cr.mass, cr.fc2_atm_num, cr.fc2_atm_indx, cr.fc2)
        self.ph0 = P.get_phonon(*args, self.irr_q, self.temps)
        self.ph = P.get_phonon(*args, self.q_pnt, self.temps)


def linewidth3_q0(st: Setup, i0, delta="gauss", sigma=0.3767, it=0, pol=None, with_w=False):
    """One pass of the q0 loop body (``main.f90:560-587``) for q0 = i0 (0-based)."""
    A, perm, cnt = momentum3(st.mesh, st.q_pnt_int, st.irr_int[i0])
    sctr = scatter_w3(st.cr, st.q_pnt, st.q_pnt_int, st.irr_int[i0], st.ph0["evec"][i0],
                      st.ph0["onebyomega"][i0], st.ph["evec"], st.ph["onebyomega"], perm)
    om0 = st.ph0["omega"][i0]
    if delta == "gauss":
        lw, p3q = lw3_gauss(om0, st.ph["omega"], st.ph["nbe"][it], sctr, A, st.q_pnt_int, sigma, pol)
        p3 = float(p3q.sum())
    else:
        lw, p3q, p3 = lw3_tetra(om0, st.ph["omega"], st.ph["nbe"][it], sctr, st.tetra, A, pol)
    out = dict(lw=lw, p3_q0=p3q, p3=p3, npairs=cnt[0])
    if with_w:
        out["sctr"] = sctr
        out["Allq1q2"] = A
        out["perm"] = perm
    return out


def linewidth3_all(st: Setup, delta="gauss", sigma=0.3767, q0_list=None, isotope=None):
    """Linewidths (nT, Nq0, Ndof) of the 3-phonon (+isotope) path for the given q0s."""
    nT = len(st.temps)
    ndof = st.cr.ndof
    q0_list = range(st.nq0) if q0_list is None else q0_list
    lw = np.zeros((nT, st.nq0, ndof))
    for i0 in q0_list:
        A, perm, cnt = momentum3(st.mesh, st.q_pnt_int, st.irr_int[i0])
        sctr = scatter_w3(st.cr, st.q_pnt, st.q_pnt_int, st.irr_int[i0], st.ph0["evec"][i0],
                          st.ph0["onebyomega"][i0], st.ph["evec"], st.ph["onebyomega"], perm)
        om0 = st.ph0["omega"][i0]
        for it in range(nT):
            if delta == "gauss":
                l3, _ = lw3_gauss(om0, st.ph["omega"], st.ph["nbe"][it], sctr, A, st.q_pnt_int, sigma)
            else:
                l3, _, _ = lw3_tetra(om0, st.ph["omega"], st.ph["nbe"][it], sctr, st.tetra, A)
            lw[it, i0] = l3
        if isotope is not None:
            wi = iso_w(st.cr.nbasis, st.ph0["evec"][i0], om0, st.ph["evec"], isotope)
            li = (iso_lw_gauss(om0, st.ph["omega"], wi, sigma) if delta == "gauss"
                  else iso_lw_tetra(om0, st.ph["omega"], wi, st.tetra))
            lw[:, i0] += 0.5 * li
    return lw


def kappa_rta(st: Setup, lw, symm=True):
    """RTA kappa (nT, 9) from linewidths (nT, Nq0, Ndof)."""
    out = []
    for it, T in enumerate(st.temps):
        if symm:
            krn = velkron_symm(st.ph0["grp_vel"], st.Rxyz, st.mult)
            out.append(kappa_symm(st.nq, st.irr_int, st.ph0["omega"], st.ph0["nbe"][it], lw[it], krn,
                                  st.cr.vol, T))
        else:
            out.append(kappa_full(st.q_pnt_int, st.pos, st.ph["omega"], st.ph["nbe"][it], st.ph["grp_vel"],
                                  lw[it], st.cr.vol, T))
    return np.array(out)


# ----------------------------------------------------------------------------- iterative BTE
def time_reversal_set(mesh, q_pnt_int):
    """Irreducible set under q ~ -q (kappa_iter.x, Irr_q_point_m.f90:216-335) with the smaller grid
    index as representative.  Returns (irr_grid, pos_tr, sgn_tr, neg, deg)."""
    mesh = np.asarray(mesh)
    neg_int = -np.asarray(q_pnt_int)
    m = np.mod(neg_int, mesh[None, :])
    neg = (m[:, 0] + mesh[0] * (m[:, 1] + mesh[1] * m[:, 2])).astype(np.int32)
    g = np.arange(len(q_pnt_int))
    rep = np.minimum(g, neg)
    irr_grid = np.unique(rep).astype(np.int32)
    pos = np.searchsorted(irr_grid, rep).astype(np.int32)
    sgn = np.where(g == rep, 1, -1).astype(np.int32)
    deg = np.bincount(pos, minlength=len(irr_grid)).astype(np.int32)
    return irr_grid, pos, sgn, neg, deg


def partner_map(mesh, q_pnt_int, q0_int):
    """kappa.x's partner p(q1) = grid(-q0 - q1) (0-based)."""
    mesh = np.asarray(mesh)
    m = np.mod(-(np.asarray(q0_int)[None, :] + np.asarray(q_pnt_int)), mesh[None, :])
    return (m[:, 0] + mesh[0] * (m[:, 1] + mesh[1] * m[:, 2])).astype(np.int32)


def bte_iter(st: Setup, it=0, eps_k=1e-6, max_iter=1000):
    """kappa_iter.x on the grid phonons of ``st`` at temperature index ``it``."""
    irr_grid, pos, sgn, neg, deg = time_reversal_set(st.mesh, st.q_pnt_int)
    nirr = len(irr_grid)
    nd = st.cr.ndof
    sctr = np.zeros((nirr, st.nq, nd, nd, nd))
    part = np.zeros((nirr, st.nq), np.int32)
    for i, g0 in enumerate(irr_grid):
        q0 = st.q_pnt_int[g0]
        A, perm, _ = momentum3(st.mesh, st.q_pnt_int, q0)
        sctr[i] = scatter_w3(st.cr, st.q_pnt, st.q_pnt_int, q0, st.ph["evec"][g0], st.ph["onebyomega"][g0],
                             st.ph["evec"], st.ph["onebyomega"], perm)
        part[i] = partner_map(st.mesh, st.q_pnt_int, q0)
    inv_tau = np.zeros((nirr, nd))
    F = np.zeros((nirr, nd, 3))
    krta = np.zeros(9)
    kap = np.zeros(9)
    iters = lib().orc_bte_iter(nd, st.nq, _i(st.tetra), nirr, irr_grid, pos, sgn, neg, part, _f(sctr),
                               _f(st.ph["omega"]), _f(st.ph["nbe"][it]), _f(st.ph["grp_vel"]), deg,
                               float(st.temps[it]), st.cr.vol, eps_k, max_iter, inv_tau, F, krta, kap)
    return dict(kappa=kap, kappa_rta=krta, inv_tau=inv_tau, F=F, iters=iters, irr_grid=irr_grid, deg=deg)


def bte_iter_gauss(st: Setup, sigma, it=0, eps_k=1e-6, max_iter=1000):
    """The iterative BTE with Gaussian delta weights (build-side form) on the grid phonons of ``st``."""
    irr_grid, pos, sgn, neg, deg = time_reversal_set(st.mesh, st.q_pnt_int)
    nirr = len(irr_grid)
    nd = st.cr.ndof
    sctr = np.zeros((nirr, st.nq, nd, nd, nd))
    part = np.zeros((nirr, st.nq), np.int32)
    for i, g0 in enumerate(irr_grid):
        q0 = st.q_pnt_int[g0]
        A, perm, _ = momentum3(st.mesh, st.q_pnt_int, q0)
        sctr[i] = scatter_w3(st.cr, st.q_pnt, st.q_pnt_int, q0, st.ph["evec"][g0], st.ph["onebyomega"][g0],
                             st.ph["evec"], st.ph["onebyomega"], perm)
        part[i] = partner_map(st.mesh, st.q_pnt_int, q0)
    inv_tau = np.zeros((nirr, nd))
    F = np.zeros((nirr, nd, 3))
    krta = np.zeros(9)
    kap = np.zeros(9)
    iters = lib().orc_bte_iter_gauss(nd, st.nq, float(sigma), nirr, irr_grid, pos, sgn, neg, part, _f(sctr),
                                     _f(st.ph["omega"]), _f(st.ph["nbe"][it]), _f(st.ph["grp_vel"]), deg,
                                     float(st.temps[it]), st.cr.vol, eps_k, max_iter, inv_tau, F, krta, kap)
    return dict(kappa=kap, kappa_rta=krta, inv_tau=inv_tau, F=F, iters=iters, irr_grid=irr_grid, deg=deg)


# ----------------------------------------------------------------------------- point defect
def _lpd():
    L = lib()
    if not hasattr(L, "_pd_set"):
        L.orc_pd_coeff.argtypes = [ct.c_double, f64p, i32p, f64p, f64p]
        L.orc_pd_coeff.restype = None
        L.orc_pd_perturbation.argtypes = [ct.c_int, ct.c_int, i32p, i32p, f64p, ct.c_int, i32p, i32p, f64p, f64p, f64p,
                                          f64p, f64p]
        L.orc_pd_perturbation.restype = None
        L.orc_pd_rate.argtypes = [ct.c_int, ct.c_int, i32p, f64p, c128p, f64p, c128p, ct.c_int, f64p, f64p,
                                  ct.c_double, ct.c_double, ct.c_int, ct.c_int, f64p]
        L.orc_pd_rate.restype = None
        L._pd_set = True
    return L


def pd_coeff(E, W, v=(0, 1, 2, 3)):
    """CoefAtVertOfTetrhd: (sorted W, vertex order, Coeff = d - i pi c) for one tetrahedron."""
    W = _f(W).copy()
    v = _i(v).copy()
    re = np.zeros(4)
    im = np.zeros(4)
    _lpd().orc_pd_coeff(float(E), W, v, re, im)
    return W, v, re + 1j * im


def pd_perturbation(cr, num_p, idx_p, fc_p, mass_def):
    """PerturbationMatrix: (V_FC, V_M) as Fortran-order (Ndof, Ndof) arrays, [col][row] in memory."""
    n = cr.ndof
    vfc = np.zeros(n * n)
    vm = np.zeros(n * n)
    _lpd().orc_pd_perturbation(cr.nbasis, cr.fc2_atm_indx.shape[1], _i(cr.fc2_atm_num), _i(cr.fc2_atm_indx),
                               _f(cr.fc2), idx_p.shape[1], _i(num_p), _i(idx_p), _f(fc_p), _f(cr.mass), _f(mass_def),
                               vfc, vm)
    return vfc, vm


def pd_rates(st: Setup, qmesh_pd, num_p, idx_p, fc_p, mass_def, rho, mat_inv_full=True, optc_therm=True, ewald=None):
    """ScatterRatePointDefect for every irreducible q0 of ``st``: (Nq0, Ndof) rates."""
    from . import phonons as Ph
    cr = st.cr
    qi, qf, tet = make_tetrahedron(qmesh_pd, cr.G, zero_centered=True)
    ph = Ph.get_phonon(cr.latvec, cr.mass, cr.fc2_atm_num, cr.fc2_atm_indx, cr.fc2, qf, [300.0], ewald=ewald)
    w2 = _f(ph["omega"] ** 2)
    vfc, vm = pd_perturbation(cr, num_p, idx_p, fc_p, mass_def)
    n = cr.ndof
    out = np.zeros((st.nq0, n))
    for i in range(st.nq0):
        g0 = int(np.all(st.irr_int[i] == 0))
        r = np.zeros(n)
        _lpd().orc_pd_rate(n, qi.shape[0], _i(tet), w2, _c(ph["evec"]), _f(st.ph0["omega"][i]), _c(st.ph0["evec"][i]),
                           g0, vfc, vm, float(rho), cr.vol, int(mat_inv_full), int(optc_therm), r)
        out[i] = r
    return out


# ----------------------------------------------------------------------------- four-phonon
def _l4():
    L = lib()
    if not hasattr(L, "_w4_set"):
        L.orc_w4_naive.argtypes = [ct.c_int, ct.c_int, i32p, i32p, f64p, f64p, f64p, ct.c_int, f64p, f64p, f64p, i32p,
                                   c128p, f64p, c128p, f64p, c128p, f64p, c128p, f64p, f64p]
        L.orc_w4_naive.restype = None
        L.orc_w4_factored.argtypes = [ct.c_int, ct.c_int, i32p, i32p, f64p, f64p, f64p, ct.c_int, f64p, i32p, i32p,
                                      c128p, f64p, c128p, f64p, ct.c_longlong, i32p, f64p]
        L.orc_w4_factored.restype = None
        L.orc_lw4_tetra.argtypes = [ct.c_int, ct.c_int, i32p, f64p, f64p, f64p, f64p, i32p, i32p, f64p, i32p, f64p]
        L.orc_lw4_tetra.restype = None
        L.orc_lw4_gauss.argtypes = [ct.c_int, ct.c_int, i32p, f64p, f64p, f64p, f64p, i32p, f64p, i32p, ct.c_double,
                                    f64p]
        L.orc_lw4_gauss.restype = None
        L._w4_set = True
    return L


def fc4_derived(cr):
    idx = cr.fc4_atm_indx
    return _i(idx[:, :, 3]), _f(np.einsum("ij,mnj->mni", cr.latvec, idx[:, :, :3].astype(np.float64)))


def w4_naive(cr, nq, q1, q2, q3, q0chk, e0, o0, e1, o1, e2, o2, e3, o3):
    """ScatterMatEl4 + ScatterProbability4 in the reference loop order, one quartet."""
    nd = cr.ndof
    btyp, posr = fc4_derived(cr)
    W = np.zeros((nd, nd, nd, nd))
    _l4().orc_w4_naive(cr.nbasis, cr.fc4.shape[1], _i(cr.fc4_atm_num), btyp, posr, _f(cr.fc4),
                       _f(1.0 / np.sqrt(cr.mass)), nq, _f(q1), _f(q2), _f(q3), _i(q0chk), _c(e0), _f(o0), _c(e1),
                       _f(o1), _c(e2), _f(o2), _c(e3), _f(o3), W)
    return W


def w4_factored(st, i0, quartets, q0_from_grid=None):
    """W4 [quartet][s0][s1][s2][s3] for 1-based grid quartets (q1, q2, q3) of q0 = irreducible i0."""
    cr = st.cr
    nd = cr.ndof
    btyp, posr = fc4_derived(cr)
    quartets = _i(quartets)
    out = np.zeros((len(quartets), nd, nd, nd, nd))
    _l4().orc_w4_factored(cr.nbasis, cr.fc4.shape[1], _i(cr.fc4_atm_num), btyp, posr, _f(cr.fc4),
                          _f(1.0 / np.sqrt(cr.mass)), st.nq, _f(st.q_pnt), _i(st.q_pnt_int), _i(st.irr_int[i0]),
                          _c(st.ph0["evec"][i0]), _f(st.ph0["onebyomega"][i0]), _c(st.ph["evec"]),
                          _f(st.ph["onebyomega"]), len(quartets), quartets, out)
    return out


def lw4_tetra(st, i0, it=0, pol=None):
    """Four-phonon scattering rate of q0 = irreducible i0 (TetrahedronIntegration4th)."""
    nd = st.cr.ndof
    if pol is None:
        pol = np.array([[1, nd]] * 4, np.int32)
    A, perm, cnt = momentum4(st.mesh, st.q_pnt_int, st.irr_int[i0])
    Wq = w4_factored(st, i0, perm)
    rate = np.zeros(nd)
    _l4().orc_lw4_tetra(nd, st.nq, _i(st.irr_int[i0]), _f(st.ph0["omega"][i0]), _f(st.ph0["nbe"][it][i0]),
                        _f(st.ph["omega"]), _f(st.ph["nbe"][it]), _i(st.tetra), _i(A), _f(Wq), _i(pol), rate)
    return rate, dict(Allq1q2q3=A, perm=perm, counts=cnt)


def q3_map(st, q0_int):
    """grid index (0-based) of q3 = -q0 - q1 - q2 for every ordered (q1, q2)."""
    mesh = st.mesh
    s = -(np.asarray(q0_int)[None, None, :] + st.q_pnt_int[:, None, :] + st.q_pnt_int[None, :, :])
    m = np.mod(s, mesh[None, None, :])
    return (m[..., 0] + mesh[0] * (m[..., 1] + mesh[1] * m[..., 2])).astype(np.int32)


def lw4_gauss(st, i0, it=0, sigma=0.3767, pol=None):
    """Gaussian four-phonon scattering rate of q0 = irreducible i0 (build-side extension)."""
    nd = st.cr.ndof
    if pol is None:
        pol = np.array([[1, nd]] * 4, np.int32)
    q3 = q3_map(st, st.irr_int[i0])
    g = np.arange(st.nq, dtype=np.int32)
    quart = np.stack([np.repeat(g, st.nq), np.tile(g, st.nq), q3.ravel()], axis=1) + 1
    W4 = w4_factored(st, i0, quart)
    rate = np.zeros(nd)
    _l4().orc_lw4_gauss(nd, st.nq, _i(st.irr_int[i0]), _f(st.ph0["omega"][i0]), _f(st.ph0["nbe"][it][i0]),
                        _f(st.ph["omega"]), _f(st.ph["nbe"][it]), _i(q3), _f(W4), _i(pol), float(sigma), rate)
    return rate


# ----------------------------------------------------------------------------- LineWidth.x path mode
def path_points(G, q_high_sym):
    """q_points_highsymm (src/LineWidth/Src/CreateMesh_mod.f90:85-172): (qpoints, dist, zero_centered)."""
    qhs = np.asarray(q_high_sym, np.float64)  # (n_nodes, 4)
    G = np.asarray(G, np.float64)
    qs, ds, zs = [], [], []
    sd = dist = 0.0
    for nd in range(len(qhs) - 1):
        a, b = qhs[nd, :3], qhs[nd + 1, :3]
        npt = int(qhs[nd + 1, 3])
        zc = bool(np.any(a < 0.0) or np.any(b < 0.0) or np.all(np.abs(a) <= 0.5) or np.all(np.abs(b) <= 0.5))
        s = np.array([G[r, 0] * a[0] + G[r, 1] * a[1] + G[r, 2] * a[2] for r in range(3)])
        e = np.array([G[r, 0] * b[0] + G[r, 1] * b[1] + G[r, 2] * b[2] for r in range(3)])
        d = e - s
        vlen = np.sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
        vh = d / vlen
        step = vlen / npt if npt != 0 else 0.0
        for ii in range(1, npt + 1):
            dist = sd + ii * step
            qs.append(s + (ii * step) * vh)
            ds.append(dist)
            zs.append(zc)
        sd = dist
    return np.array(qs).reshape(-1, 3), np.array(ds), np.array(zs, bool)


def _lpath():
    L = lib()
    if not hasattr(L, "_path_set"):
        L.orc_w3_path.argtypes = [ct.c_int, ct.c_int, i32p, i32p, f64p, f64p, f64p, ct.c_int, ct.c_int, f64p, f64p,
                                  i32p, c128p, f64p, c128p, f64p, c128p, f64p, f64p]
        L.orc_w3_path.restype = None
        L.orc_lw_path_tetra.argtypes = [ct.c_int, ct.c_int, f64p, f64p, f64p, f64p, f64p, f64p, i32p, f64p]
        L.orc_lw_path_tetra.restype = None
        L.orc_lw_path_gauss.argtypes = [ct.c_int, ct.c_int, f64p, f64p, f64p, f64p, f64p, f64p, i32p, i32p,
                                        ct.c_double, f64p]
        L.orc_lw_path_gauss.restype = None
        L._path_set = True
    return L


def find_q2(G, q0, q1s, zero_centered):
    """q2 = G - (q0 + q1) for the first G of (0,1,-1,2,-2)^3 (first component fastest) inside the zone,
    tested in fractional coordinates from LAPACK's LU solve (ScatterProbAllq1 / CheckIfWithinBZ,
    Linewidth_m.f90:115-185, 458-497).  Returns (q2 (n, 3), exists (n,))."""
    import scipy.linalg as sl
    G = np.asarray(G, np.float64)
    lu = sl.lu_factor(G)
    sgn = [0, 1, -1, 2, -2]
    n = len(q1s)
    q2 = np.zeros((n, 3))
    found = np.zeros(n, bool)
    base = np.asarray(q0)[None, :] + np.asarray(q1s)
    for c3 in sgn:
        for c2 in sgn:
            for c1 in sgn:
                idx = np.array([c1, c2, c3], np.float64)
                gv = np.array([G[r, 0] * idx[0] + G[r, 1] * idx[1] + G[r, 2] * idx[2] for r in range(3)])
                t = gv[None, :] - base
                x = sl.lu_solve(lu, t.T).T
                if zero_centered:
                    inside = np.all(np.abs(x) <= 0.5, axis=1)
                else:
                    inside = np.all(x >= 0.0, axis=1) & np.all(x <= 1.0, axis=1)
                take = inside & ~found
                q2[take] = t[take]
                found |= take
    return q2, found


def linewidth_path(st: Setup, q0, zero_centered, delta="tetra", sigma=0.3767, it=0, q0_phonons=None):
    """LineWidth.x linewidth at one off-grid q0 (Cartesian), one temperature: ScatterProbAllq1 +
    CalculateLwTetrahedron / CalculateLinewidth.  The q1 mesh is the setup's grid; non-zero-centred
    segments use the [0, N) vectors of the same grid points and their phonons."""
    cr = st.cr
    nd = cr.ndof
    args = (cr.latvec, cr.mass, cr.fc2_atm_num, cr.fc2_atm_indx, cr.fc2)
    ph0 = q0_phonons if q0_phonons is not None else P.get_phonon(*args, np.asarray(q0)[None, :], st.temps)
    if zero_centered:
        q1s = st.q_pnt
    else:
        _, q1s, _ = make_tetrahedron(st.mesh, st.cr.G, zero_centered=False)
    q2, ex = find_q2(st.cr.G, q0, q1s, zero_centered)
    ph2 = P.get_phonon(*args, q2, st.temps)
    ph2["omega"][~ex] = 0.0
    ph2["nbe"][:, ~ex] = 0.0
    q0chk = np.stack([np.full(st.nq, np.all(np.abs(q0) < C.zero_prec)),
                      np.all(st.q_pnt_int == 0, axis=1),
                      np.all(np.abs(q2) < C.zero_prec, axis=1)], axis=1).astype(np.int32)
    btyp, posr = fc3_derived(cr)
    W = np.zeros((st.nq, nd, nd, nd))
    _lpath().orc_w3_path(cr.nbasis, cr.fc3.shape[1], _i(cr.fc3_atm_num), btyp, posr, _f(cr.fc3), _f(cr.mass),
                         st.nq, st.nq, _f(q1s), _f(q2), _i(q0chk), _c(ph0["evec"][0]), _f(ph0["omega"][0]),
                         _c(st.ph["evec"]), _f(st.ph["omega"]), _c(ph2["evec"]), _f(ph2["omega"]), W)
    W[~ex] = 0.0
    lw = np.zeros(nd)
    if delta == "tetra":
        _lpath().orc_lw_path_tetra(nd, st.nq, _f(ph0["omega"][0]), _f(st.ph["omega"]), _f(st.ph["nbe"][it]),
                                   _f(ph2["omega"]), _f(ph2["nbe"][it]), _f(W), _i(st.tetra), lw)
    else:
        _lpath().orc_lw_path_gauss(nd, st.nq, _f(ph0["omega"][0]), _f(st.ph["omega"]), _f(st.ph["nbe"][it]),
                                   _f(ph2["omega"]), _f(ph2["nbe"][it]), _f(W), _i(ex.astype(np.int32)),
                                   _i(st.q_pnt_int), float(sigma), lw)
    return lw, dict(omega0=ph0["omega"][0], q2=q2, exists=ex, W=W)
