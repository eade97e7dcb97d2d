"""Oracle (test infrastructure only): harmonic phonons in FP64 with LAPACK zheevd.

CPU restatement of ``get_phonon`` (``src/Kappa/Src/DynaMat_mod.f90:486-709``)
with ``DynMatgv_SR`` (``DynaMat_mod.f90:98-190``) and ``SolveEigen``
(``src/Kappa/Src/lapack_gfort.f90:212-265``).  ``numpy.linalg.eigh`` with
``UPLO='U'`` calls LAPACK ``zheevd('V','U')`` exactly as the reference does,
so eigenvalue order and eigenvector gauge follow the same library routine.
With ``ewald`` (an :class:`oracle.ewald.Ewald`) the ``LongEw`` branch adds the
dipole-dipole matrix and its q-derivative (``DynaMat_mod.f90:548-590``).

Only ``tests/``, ``bench.py``'s CPU-baseline leg and ``__graft_entry__.smoke``
may import this module; the product never does.
"""
from __future__ import annotations

import numpy as np

from . import constants as C


def dynmat(latvec, mass, atm_num, atm_indx, fc2, q):
    """D(q) and dD/dq_k (``DynMatgv_SR``, ``DynaMat_mod.f90:98-190``)."""
    nb = len(mass)
    ndof = 3 * nb
    D = np.zeros((ndof, ndof), dtype=np.complex128)
    dD = np.zeros((3, ndof, ndof), dtype=np.complex128)
    for mu in range(nb):
        for n in range(int(atm_num[mu])):
            R = atm_indx[mu, n, :3].astype(np.float64)
            nu = int(atm_indx[mu, n, 3]) - 1
            Rxyz = latvec @ R
            ph = np.exp(1j * np.dot(q, Rxyz))
            mf = 1.0 / np.sqrt(mass[mu] * mass[nu])
            blk = fc2[mu, n, :, :, 0] * ph * mf          # [alpha, beta]
            D[3 * mu:3 * mu + 3, 3 * nu:3 * nu + 3] += blk
            for k in range(3):
                dD[k, 3 * mu:3 * mu + 3, 3 * nu:3 * nu + 3] += blk * 1j * Rxyz[k]
    return D, dD


def get_phonon(latvec, mass, atm_num, atm_indx, fc2, qpoints, temps, ewald=None, gamma_dir=None):
    """Per q: omega (rad/ps), 1/(omega wTHz), nBE per T, group velocity, eigenvectors.

    ``qpoints`` is (Nq, 3) Cartesian.  Returns a dict of arrays in
    Fortran-compatible C-order layouts:
    ``evec (Nq, Ndof(s), Ndof(row))`` (i.e. Fortran ``Evec(row, s, q)``),
    ``omega (Nq, Ndof)``, ``onebyomega (Nq, Ndof)``, ``nbe (nT, Nq, Ndof)``,
    ``grp_vel (Nq, Ndof, 3)``.
    """
    qpoints = np.asarray(qpoints, dtype=np.float64)
    temps = np.atleast_1d(np.asarray(temps, dtype=np.float64))
    nq = qpoints.shape[0]
    ndof = 3 * len(mass)
    evec = np.zeros((nq, ndof, ndof), dtype=np.complex128)
    omega = np.zeros((nq, ndof))
    oneby = np.zeros((nq, ndof))
    nbe = np.zeros((len(temps), nq, ndof))
    vel = np.zeros((nq, ndof, 3))
    for i in range(nq):
        q = qpoints[i]
        D, dD = dynmat(latvec, mass, atm_num, atm_indx, fc2, q)
        if ewald is not None:
            De, dDe = ewald.term(qpoints, i, mass, gamma_dir)
            D = D + De
            dD = dD + dDe
        w, v = np.linalg.eigh(D, UPLO="U")
        neg = (np.abs(w) > C.EPS) & (w < 0.0)
        W = np.sqrt(np.abs(w))
        W[neg] *= -1.0
        strt = 3 if np.all(np.abs(q) < C.cmp_prec) else 0
        for df in range(strt, ndof):
            om = W[df]
            e = v[:, df]
            cv = np.array([np.vdot(e, dD[k] @ e) for k in range(3)]) / (2.0 * om)
            vel[i, df] = cv.real * C.vg_ms
            for it, T in enumerate(temps):
                nbe[it, i, df] = 1.0 / (np.exp(C.BEConv * abs(om) / T) - 1.0)
            oneby[i, df] = 1.0 / (om * C.wTHz)
        omega[i] = W * C.wTHz
        evec[i] = v.T          # evec[q, s, row] = Evec(row, s, q)
    return dict(evec=evec, omega=omega, onebyomega=oneby, nbe=nbe, grp_vel=vel)
