"""Oracle (test infrastructure only): the Ewald dipole-dipole part of the dynamical matrix.

CPU restatement, in the reference's loop order, of

- ``set_EwaldParam`` / ``DecideEwaldParameters`` / ``ConstTerm`` / ``SumRule``
  (``src/Kappa/Src/EwaldParam.f90``), with ``mesh_points`` (``CreateMesh_mod.f90:32-83``)
  and ``fold_indx`` (``IndxChng_mod.f90:85-107``);
- ``RealSpaceEW(_gv)``, ``H_func``, ``KSpaceEW(_gv)``, ``CombineZStar(_gv)``
  (``src/Kappa/Src/EwaldSum_mod.f90:37-563``);
- ``DynMat_Ew``, ``DynMatgv_Ew``, ``DynMat_NA`` (``src/Kappa/Src/DynaMat_mod.f90:193-483``)
  and the ``LongEw`` branch of ``get_phonon`` (``DynaMat_mod.f90:548-590``), with the
  fixed Gamma direction of ``get_phonon_singleq`` (``src/LineWidth/Src/DynaMat_mod.f90:770-800``).

Array conventions: ``C[mu, nu][alpha, beta]`` is Fortran ``C(beta, alpha, nu, mu)``;
matrices are indexed as in Fortran, ``Z[mu][i, j]`` = ``Zstar(i, j, mu)``, ``eps[i, j]`` =
``eps(i, j)``; lattice and reciprocal vectors are the columns of ``latvec`` and ``G`` (as in the
synthetic crystal).  Only ``tests/`` may import this module.
"""
from __future__ import annotations

import math

import numpy as np

from . import constants as C

# ((1.602176634 * 2.99792458)**2 * 6.241509074460763 * 0.1): e^2 / (4 pi eps0) in eV A
eV_A2 = (1.602176634 * 2.99792458) ** 2 * 6.241509074460763 * 0.1
QDIR_SINGLE = np.array([0.0034, 0.0, 0.001234])   # get_phonon_singleq's Gamma direction


def fold_indx(dimen, indx):
    out = list(indx)
    for k in range(3):
        if out[k] > dimen[k] // 2:
            out[k] -= dimen[k]
    return out


def mesh_points(cell_vec, mesh):
    """Zero-centred, undivided mesh (``mesh_points(cell, mesh, .false., .true.)``): rows = points,
    i1 outermost, i3 innermost."""
    pts = []
    for i1 in range(mesh[0]):
        for i2 in range(mesh[1]):
            for i3 in range(mesh[2]):
                f = fold_indx(mesh, (i1, i2, i3))
                pts.append(cell_vec @ np.array(f, np.float64))
    return np.array(pts)


def decide_parameters(eps, eps_inv, latvec, G, sup_cell, prec_ew):
    """``DecideEwaldParameters``: (Lmb, NKcut)."""
    p = -math.log(prec_ew)
    ncut = np.array([sup_cell[0] // 2 + 1, 0, 0], np.float64)
    rcut = latvec @ ncut
    delv = rcut @ eps_inv           # matmul(dV, eps_inv): sum_i dV(i) eps_inv(i, j)
    D = math.sqrt(float(np.dot(delv, rcut)))
    lmb = math.sqrt(p) / D
    normG = float(np.linalg.norm(G[:, 0]))
    kcut = 2.0 * p / (D * math.sqrt((eps[0, 0] + eps[1, 1] + eps[2, 2]) / 3.0))
    return lmb, int(math.ceil(kcut / normG))


def h_func(ld):
    cerfn = math.erfc(ld)
    y2 = ld * ld
    invy2 = 1.0 / y2
    invy3 = invy2 / ld
    pe = (2.0 / math.sqrt(C.PI)) * math.exp(-y2)
    h1 = (3.0 * invy3 * cerfn + pe * (3.0 * invy2 + 2.0)) * invy2
    h2 = cerfn * invy3 + pe * invy2
    return h1, h2


class Ewald:
    """``EwaldParam`` for one cell.  ``eps`` and ``zstar`` in the conventions above; ``tau`` the
    Cartesian basis positions (Nb, 3)."""

    def __init__(self, latvec, G, vol, tau, eps, zstar, rmesh, decide=True, prec_ew=1e-6, lmb=0.8,
                 gmesh=None, sup_cell=(5, 5, 5)):
        self.latvec, self.G, self.vol = np.asarray(latvec, float), np.asarray(G, float), float(vol)
        self.tau = np.asarray(tau, float)
        self.eps = np.asarray(eps, float)
        self.Z = np.asarray(zstar, float)
        self.nb = self.tau.shape[0]
        # eps_inv = transpose(inverse(transpose(eps))) = inverse(eps)
        self.eps_inv = np.linalg.inv(self.eps)
        self.det = float(np.linalg.det(self.eps))
        if decide:
            self.lmb, nk = decide_parameters(self.eps, self.eps_inv, self.latvec, self.G, sup_cell, prec_ew)
            self.gmesh = [2 * nk + 1] * 3
        else:
            self.lmb, self.gmesh = float(lmb), list(gmesh)
        self.rmesh = list(rmesh)
        self.R = mesh_points(self.latvec, self.rmesh)
        self.Gp = mesh_points(self.G, self.gmesh)
        nb = self.nb
        cconst = np.zeros((nb, nb, 3, 3), np.complex128)
        cnst = 4.0 * self.lmb ** 3 / (3.0 * math.sqrt(C.PI) * math.sqrt(self.det))
        for mu in range(nb):
            cconst[mu, mu] = self.eps_inv.T * cnst      # CConst(beta, alpha) = eps_inv(beta, alpha)
        self.cconst = cconst
        cq0 = self.k_space(np.zeros(3)) - self.real_space(np.zeros(3)) - cconst
        cq0z = self.combine(cq0)
        self.csum = cq0z.sum(axis=1)                    # CSumq0(beta, alpha, mu) = sum_nu Cq0Z

    # ---- EwaldSum_mod
    def real_space(self, q, grad=False):
        nb = self.nb
        out = np.zeros((nb, nb, 3, 3), np.complex128)
        dout = np.zeros((3, nb, nb, 3, 3), np.complex128)
        for R in self.R:
            expn = np.exp(1j * float(np.dot(q, R)))
            for mu in range(nb):
                for nu in range(nb):
                    if np.all(np.abs(R) < C.cmp_prec) and mu == nu:
                        continue
                    dV = R + self.tau[nu] - self.tau[mu]
                    delV = dV @ self.eps_inv            # sum_i dV(i) eps_inv(i, j)
                    DC = math.sqrt(float(np.dot(delV, dV)))
                    delV = self.lmb * delV
                    h1, h2 = h_func(self.lmb * DC)
                    hab = np.outer(delV, delV) * h1 - self.eps_inv.T * h2   # [alpha, beta]: eps_inv(beta, alpha)
                    out[mu, nu] += expn * hab
                    if grad:
                        for k in range(3):
                            dout[k, mu, nu] += 1j * R[k] * expn * hab
        s = self.lmb ** 3 / math.sqrt(self.det)
        return (out * s, dout * s) if grad else out * s

    def k_space(self, q, grad=False):
        nb = self.nb
        out = np.zeros((nb, nb, 3, 3), np.complex128)
        dout = np.zeros((3, nb, nb, 3, 3), np.complex128)
        eps = self.eps
        for G in self.Gp:
            if not (np.any(np.abs(q) > C.cmp_prec) or np.any(np.abs(G) > C.cmp_prec)):
                continue
            K = G + q
            eK = K @ eps                                # matmul(K, eps): sum_i K(i) eps(i, j)
            KeK = float(np.dot(K, eK))
            KG = math.exp(-KeK / (4.0 * self.lmb ** 2)) / KeK
            if grad:
                epsK = np.array([np.dot(eps[:, i], K) + np.dot(K, eps[i, :]) for i in range(3)])
                KpLmb = 1.0 / KeK + 0.25 / self.lmb ** 2
            for mu in range(nb):
                for nu in range(nb):
                    tmn = self.tau[mu] - self.tau[nu]
                    Kmn = KG * np.exp(1j * float(np.dot(K, tmn)))
                    Kab = np.outer(K, K) * Kmn          # [alpha, beta]
                    out[mu, nu] += Kab
                    if grad:
                        for k in range(3):
                            kmat = np.zeros((3, 3))
                            kmat[k, :] += K             # d(K_alpha K_beta)/dK_k
                            kmat[:, k] += K
                            dout[k, mu, nu] += Kab * (1j * tmn[k] - epsK[k] * KpLmb) + Kmn * kmat
        s = 4.0 * C.PI / self.vol
        return (out * s, dout * s) if grad else out * s

    def combine(self, Cq):
        """CombineZStar: CqZ(b, a, nu, mu) = sum Z(ap, a, mu) Z(bp, b, nu) Cq(bp, ap, nu, mu)."""
        nb = self.nb
        out = np.zeros_like(Cq)
        for mu in range(nb):
            for nu in range(nb):
                # Z[mu][ap, a] = Zstar(ap, a, mu); Cq[mu, nu][ap, bp] = Cq(bp, ap, nu, mu)
                out[mu, nu] = self.Z[mu].T @ Cq[mu, nu] @ self.Z[nu]
        return out

    # ---- DynaMat_mod
    def _to_dyn(self, CqZ, mass):
        nb = self.nb
        D = np.zeros((3 * nb, 3 * nb), np.complex128)
        for mu in range(nb):
            for nu in range(nb):
                D[3 * mu:3 * mu + 3, 3 * nu:3 * nu + 3] = CqZ[mu, nu] / math.sqrt(mass[mu] * mass[nu])
        return D

    def dynmat(self, q, mass, grad=False):
        """DynMat_Ew / DynMatgv_Ew: D_ew (Ndof, Ndof) and (grad) dD_ew (3, Ndof, Ndof)."""
        if grad:
            cr, dcr = self.real_space(q, True)
            ck, dck = self.k_space(q, True)
        else:
            cr, ck = self.real_space(q), self.k_space(q)
        cqz = self.combine(ck - cr - self.cconst)
        for mu in range(self.nb):
            cqz[mu, mu] -= self.csum[mu]
        D = self._to_dyn(cqz * eV_A2, mass)
        if not grad:
            return D
        dD = np.array([self._to_dyn(self.combine(dck[k] - dcr[k]) * eV_A2, mass) for k in range(3)])
        return D, dD

    def dynmat_na(self, qhat, mass):
        """DynMat_NA: the q = 0 Ewald matrix plus the non-analytic term along qhat."""
        D0 = self.dynmat(np.zeros(3), mass)
        nb = self.nb
        NA = np.zeros_like(D0)
        for nu in range(nb):
            for be in range(3):
                t2 = float(np.dot(qhat, self.Z[nu][be, :]))   # dot_product(q, Zstar(beta, :, nu))
                for mu in range(nb):
                    for al in range(3):
                        t1 = float(np.dot(qhat, self.Z[mu][al, :]))
                        NA[3 * mu + al, 3 * nu + be] = t1 * t2 / math.sqrt(mass[mu] * mass[nu])
        denom = float(np.dot(qhat, qhat @ self.eps))
        return D0 + NA * 4.0 * C.PI * eV_A2 / (self.vol * denom)

    def term(self, qpoints, i, mass, gamma_dir=None):
        """The LongEw addition of get_phonon for point i of the list: (D_ew, dD_ew)."""
        q = qpoints[i]
        if np.all(np.abs(q) < C.cmp_prec):
            if gamma_dir is not None:
                qhat = q + gamma_dir
            elif i != len(qpoints) - 1:
                qhat = qpoints[i + 1] - qpoints[i]
            else:
                qhat = qpoints[i] - qpoints[i - 1]
            h = float(np.linalg.norm(qhat)) / 8.0
            D = self.dynmat_na(qhat, mass)
            dD = np.zeros((3,) + D.shape, np.complex128)
            for k in range(3):
                dq = np.zeros(3)
                dq[k] = 0.5 * h
                dD[k] = (self.dynmat(q + dq, mass) - self.dynmat(q - dq, mass)) / h
            return D, dD
        return self.dynmat(q, mass, grad=True)
