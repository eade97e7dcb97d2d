"""Seeded synthetic crystals and force constants in SPRING's in-memory layout.

SPRING reads its force constants from HDF5 files written by ``reconst2/3/4.x``
(``src/Kappa/Src/hdf5_wrap_mod.f90:40-337``).  No such files exist for the
benchmark crystals, so this module builds them from a spring model with seeded
noise and returns arrays with exactly the shapes and index order of the
reference's ``FC2type`` / ``FC3type`` / ``FC4type`` (``src/Kappa/Src/FC2_mod.f90:29``,
``FC3_mod.f90:30``, ``FC4_mod.f90:30``) and ``cell`` (``unit_mod.f90:29``).

Index conventions (Fortran column-major, stored here as C-order arrays with the
axes reversed, so the flat memory is identical to the Fortran array):

* ``fc2``   Fortran ``fC(1,3,3,Na2,Nb)`` = ``(1, beta, alpha, N, mu)``
  -> numpy shape ``(Nb, Na2, 3, 3, 1)`` indexed ``[mu, N, alpha, beta, 0]``.
* ``fc3``   Fortran ``fC(3,3,3,Na3,Na3,Nb)`` = ``(gamma, beta, alpha, N2, N1, mu)``
  -> numpy ``(Nb, Na3, Na3, 3, 3, 3)`` indexed ``[mu, N1, N2, alpha, beta, gamma]``.
* ``fc4``   Fortran ``fC(3,3,3,3,Na4,Na4,Na4,Nb)``
  -> numpy ``(Nb, Na4, Na4, Na4, 3, 3, 3, 3)`` indexed ``[mu, N1, N2, N3, a, b, c, d]``.
* ``atm_indx`` Fortran ``atmIndx(4, Na, Nb)`` -> numpy ``(Nb, Na, 4)``: integer
  lattice cell ``(R1, R2, R3)`` and the 1-based basis index of the neighbour.

Spring model (the benchmark crystal "fcc rocksalt, 1st+2nd neighbour
central/tangential springs k1=8, k2=1.5 eV/A^2"): for a bond with unit vector
``r`` the pair force constant is ``-(kc r r^T + kt (1 - r r^T))``.  The
tangential constant is not pinned by the workload description; this generator
uses ``kt = TANGENTIAL_FRACTION * kc`` with ``TANGENTIAL_FRACTION = 0.2``, which
keeps every mode of both cells real.  Noise is a symmetric 3x3 N(0, sigma)
matrix per bond, shared by both directions of the bond, so D(q) is Hermitian;
the on-site block is then set by the acoustic sum rule.

Third/fourth order: every neighbour slot of the 1st-shell cluster (self + 6
nearest neighbours, Na3 = Na4 = 7) gets N(0, sigma) entries; the tensor is then
projected, by alternating orthogonal projections, onto the intersection of
(i) symmetry under permutation of the neighbour slots (with their Cartesian
indices) and (ii) the acoustic sum rule over the last slot.
"""
from __future__ import annotations

import dataclasses
import numpy as np

TANGENTIAL_FRACTION = 0.2

# Default seeds (documented so that every fixture can be regenerated).
SEED_FC2 = 2
SEED_FC3 = 3
SEED_FC4 = 4


@dataclasses.dataclass
class Crystal:
    """A ``cell`` (``src/Kappa/Src/unit_mod.f90:29-52``) plus its force constants."""

    name: str
    latvec: np.ndarray          # (3,3): columns are lattice vectors (Fortran Latvec(:, i))
    basis_frac: np.ndarray      # (Nb, 3) fractional positions (Fortran atm_pos(:, i))
    typ_indx: np.ndarray        # (Nb,) 1-based species index
    mass: np.ndarray            # (Nb,) amu per basis atom
    fc2_atm_num: np.ndarray = None
    fc2_atm_indx: np.ndarray = None
    fc2: np.ndarray = None
    fc3_atm_num: np.ndarray = None
    fc3_atm_indx: np.ndarray = None
    fc3: np.ndarray = None
    fc4_atm_num: np.ndarray = None
    fc4_atm_indx: np.ndarray = None
    fc4: np.ndarray = None
    zstar: np.ndarray = None    # (Nb, 3, 3) Born charges, zstar[mu][i, j] = Fortran BornZ(i, j, mu)
    eps: np.ndarray = None      # (3, 3) high-frequency dielectric tensor, eps[i, j] = dielec(i, j)

    @property
    def nbasis(self) -> int:
        return int(self.basis_frac.shape[0])

    @property
    def ndof(self) -> int:
        return 3 * self.nbasis

    @property
    def vol(self) -> float:
        """Cell volume, ``unit_mod.f90:178-181``."""
        a = self.latvec
        return float(abs(np.dot(a[:, 0], np.cross(a[:, 1], a[:, 2]))))

    @property
    def G(self) -> np.ndarray:
        """Reciprocal vectors as columns, ``G(:,i) = 2 pi a_j x a_k / vol`` (``unit_mod.f90:193-203``)."""
        a = self.latvec
        g = np.zeros((3, 3))
        for i in range(3):
            i2, i3 = (i + 1) % 3, (i + 2) % 3
            g[:, i] = np.cross(a[:, i2], a[:, i3]) * 2.0 * np.pi / self.vol
        return g

    def tau(self) -> np.ndarray:
        """Cartesian basis positions (Nb, 3)."""
        return self.basis_frac @ self.latvec.T


def rocksalt_primitive(a: float = 4.21, masses=(24.305, 15.999)) -> Crystal:
    """fcc rocksalt primitive cell: a/2(0,1,1), a/2(1,0,1), a/2(1,1,0); cation at 0, anion at 1/2."""
    latvec = 0.5 * a * np.array([[0.0, 1.0, 1.0], [1.0, 0.0, 1.0], [1.0, 1.0, 0.0]]).T
    basis = np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.5]])
    return Crystal("rocksalt2", latvec, basis, np.array([1, 2], dtype=np.int32),
                   np.array(masses, dtype=np.float64))


def rocksalt_cubic(a: float = 4.21, masses=(24.305, 15.999)) -> Crystal:
    """8-atom simple-cubic conventional rocksalt cell (4 cations + 4 anions, Ndof = 24)."""
    latvec = a * np.eye(3)
    cat = [[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]]
    an = [[.5, 0, 0], [0, .5, 0], [0, 0, .5], [.5, .5, .5]]
    basis = np.array(cat + an, dtype=np.float64)
    typ = np.array([1] * 4 + [2] * 4, dtype=np.int32)
    mass = np.array([masses[0]] * 4 + [masses[1]] * 4, dtype=np.float64)
    return Crystal("rocksalt8", latvec, basis, typ, mass)


def _neighbour_shells(cr: Crystal, nshell: int, rng_cells: int = 2, tol: float = 1e-6):
    """Per basis atom: list of (R(3) int, nu 0-based, r_cart(3), shell) sorted self-first, then by shell."""
    tau = cr.tau()
    nb = cr.nbasis
    out = []
    for mu in range(nb):
        cands = []
        rng = range(-rng_cells, rng_cells + 1)
        for r1 in rng:
            for r2 in rng:
                for r3 in rng:
                    R = np.array([r1, r2, r3])
                    for nu in range(nb):
                        d = cr.latvec @ R + tau[nu] - tau[mu]
                        cands.append((float(np.linalg.norm(d)), (r1, r2, r3), nu, d))
        dists = sorted({round(c[0], 6) for c in cands})
        shells = dists[: nshell + 1]  # includes 0 (self)
        sel = []
        for c in cands:
            dr = round(c[0], 6)
            if dr in shells:
                sel.append((shells.index(dr), c[1], c[2], c[3]))
        sel.sort(key=lambda s: (s[0], s[1], s[2]))
        out.append([(np.array(s[1], dtype=np.int32), s[2], s[3], s[0]) for s in sel])
    return out


def _bond_key(mu, R, nu):
    """Canonical key of the bond (mu,0)-(nu,R) == (nu,0)-(mu,-R)."""
    a = (mu, tuple(int(x) for x in R), nu)
    b = (nu, tuple(-int(x) for x in R), mu)
    return min(a, b)


def make_fc2(cr: Crystal, k=(8.0, 1.5), noise=0.05, seed=SEED_FC2) -> None:
    """Spring-model FC2 on shells 1 and 2 plus symmetric per-bond noise; on-site block from the ASR."""
    nbr = _neighbour_shells(cr, 2)
    na = max(len(n) for n in nbr)
    nb = cr.nbasis
    rng = np.random.default_rng(seed)
    noise_of = {}
    fc = np.zeros((nb, na, 3, 3, 1))
    idx = np.zeros((nb, na, 4), dtype=np.int32)
    num = np.zeros(nb, dtype=np.int32)
    # deterministic order of noise draws: sorted bond keys
    keys = sorted({_bond_key(mu, R, nu) for mu in range(nb) for (R, nu, d, sh) in nbr[mu] if sh > 0})
    for kk in keys:
        m = rng.normal(0.0, noise, size=(3, 3))
        noise_of[kk] = 0.5 * (m + m.T)
    for mu in range(nb):
        num[mu] = len(nbr[mu])
        for n, (R, nu, d, sh) in enumerate(nbr[mu]):
            idx[mu, n, :3] = R
            idx[mu, n, 3] = nu + 1
            if sh == 0:
                continue
            kc = k[sh - 1]
            kt = TANGENTIAL_FRACTION * kc
            rh = d / np.linalg.norm(d)
            P = np.outer(rh, rh)
            phi = -(kc * P + kt * (np.eye(3) - P)) + noise_of[_bond_key(mu, R, nu)]
            fc[mu, n, :, :, 0] = phi
        fc[mu, 0, :, :, 0] = -fc[mu, 1:num[mu], :, :, 0].sum(axis=0)
    cr.fc2_atm_num, cr.fc2_atm_indx, cr.fc2 = num, idx, fc


def _cluster(cr: Crystal):
    nbr = _neighbour_shells(cr, 1)
    na = max(len(n) for n in nbr)
    nb = cr.nbasis
    idx = np.zeros((nb, na, 4), dtype=np.int32)
    num = np.zeros(nb, dtype=np.int32)
    for mu in range(nb):
        num[mu] = len(nbr[mu])
        for n, (R, nu, d, sh) in enumerate(nbr[mu]):
            idx[mu, n, :3] = R
            idx[mu, n, 3] = nu + 1
    return num, idx


def make_fc3(cr: Crystal, sigma=2.0, seed=SEED_FC3, iters=200) -> None:
    """Dense 1st-shell FC3, symmetric under (N1,beta)<->(N2,gamma), ASR over the last slot."""
    num, idx = _cluster(cr)
    nb, na = cr.nbasis, idx.shape[1]
    rng = np.random.default_rng(seed)
    f = rng.normal(0.0, sigma, size=(nb, na, na, 3, 3, 3))
    for _ in range(iters):
        f = 0.5 * (f + f.transpose(0, 2, 1, 3, 5, 4))
        f = f - f.mean(axis=2, keepdims=True)
    f = 0.5 * (f + f.transpose(0, 2, 1, 3, 5, 4))
    cr.fc3_atm_num, cr.fc3_atm_indx, cr.fc3 = num, idx, np.ascontiguousarray(f)


def make_fc4(cr: Crystal, sigma=5.0, seed=SEED_FC4, iters=200) -> None:
    """Dense 1st-shell FC4, symmetric under permutations of the three neighbour slots, ASR over the last."""
    num, idx = _cluster(cr)
    nb, na = cr.nbasis, idx.shape[1]
    rng = np.random.default_rng(seed)
    f = rng.normal(0.0, sigma, size=(nb, na, na, na, 3, 3, 3, 3))
    # axes: 0 mu, 1 N1, 2 N2, 3 N3, 4 a, 5 b, 6 c, 7 d ; slot k pairs (1+k) with (5+k)
    perms = []
    import itertools
    for p in itertools.permutations(range(3)):
        ax = [0] + [1 + p[i] for i in range(3)] + [4] + [5 + p[i] for i in range(3)]
        perms.append(ax)

    def sym(x):
        return sum(x.transpose(ax) for ax in perms) / 6.0

    for _ in range(iters):
        f = sym(f)
        f = f - f.mean(axis=3, keepdims=True)
    f = sym(f)
    cr.fc4_atm_num, cr.fc4_atm_indx, cr.fc4 = num, idx, np.ascontiguousarray(f)


def build(name: str = "rocksalt2", fc4: bool = False, seeds=(SEED_FC2, SEED_FC3, SEED_FC4)) -> Crystal:
    """The benchmark crystals: ``rocksalt2`` (Ndof 6) or ``rocksalt8`` (Ndof 24)."""
    cr = rocksalt_primitive() if name == "rocksalt2" else rocksalt_cubic()
    make_fc2(cr, seed=seeds[0])
    make_fc3(cr, seed=seeds[1])
    if fc4:
        make_fc4(cr, seed=seeds[2])
    return cr


def defect_fc2(cr: Crystal, site: int = 0, scale: float = 1.15):
    """The FC2 of a cell with a substitutional defect on basis atom `site`: the pristine arrays with
    that atom's on-site block scaled (the home-cell block PerturbationMatrix reads), as
    (atm_num, atm_indx, fc2) in the set_fc2 layout."""
    fc = cr.fc2.copy()
    for n in range(int(cr.fc2_atm_num[site])):
        if np.all(cr.fc2_atm_indx[site, n, :3] == 0) and cr.fc2_atm_indx[site, n, 3] == site + 1:
            fc[site, n] *= scale
    return cr.fc2_atm_num.copy(), cr.fc2_atm_indx.copy(), fc


def make_polar(cr: Crystal, z: float = 1.986, eps: float = 3.0) -> Crystal:
    """Born charges +z (species 1) / -z (species 2) times the identity and an isotropic dielectric
    tensor: the inputs of the dipole-dipole term (``&AtmInfo`` BornZ, dielec).  The default z is
    MgO's."""
    cr.zstar = np.array([(1.0 if t == 1 else -1.0) * z * np.eye(3) for t in cr.typ_indx])
    cr.eps = eps * np.eye(3)
    return cr


def point_group(cr: Crystal, symprec: float = 1e-5):
    """Rotations W (fractional, integer) of the crystal's point group.

    Restates what ``spg_get_symmetry`` provides to ``set_SpaceGrSPGlib``
    (``src/Kappa/Src/Symmetry_m.f90:46-119``) for these cells: every integer
    matrix with entries in {-1,0,1} that preserves the metric and maps the
    basis onto itself (same species) up to a translation.  Returns
    ``(W (n,3,3) int32, Rxyz (n,3,3) Cartesian)`` with ``Rxyz = L W L^-1``.
    Pure translations of non-primitive cells give repeated rotations; like
    spglib's point-group use, only distinct rotations are kept.
    """
    import itertools
    L = cr.latvec
    metric = L.T @ L
    Linv = np.linalg.inv(L)
    pos = cr.basis_frac
    rots = []
    for ent in itertools.product((-1, 0, 1), repeat=9):
        W = np.array(ent, dtype=np.int64).reshape(3, 3)
        if round(abs(np.linalg.det(W))) != 1:
            continue
        if not np.allclose(W.T @ metric @ W, metric, atol=1e-8):
            continue
        # find a translation t such that W x_i + t maps the basis onto itself
        ok = False
        Wx0 = W @ pos[0]
        for j in range(cr.nbasis):
            if cr.typ_indx[j] != cr.typ_indx[0]:
                continue
            t = pos[j] - Wx0
            good = True
            for i in range(cr.nbasis):
                y = W @ pos[i] + t
                hit = False
                for k in range(cr.nbasis):
                    if cr.typ_indx[k] != cr.typ_indx[i]:
                        continue
                    d = y - pos[k]
                    if np.allclose(d - np.round(d), 0.0, atol=symprec):
                        hit = True
                        break
                if not hit:
                    good = False
                    break
            if good:
                ok = True
                break
        if ok:
            rots.append(W)
    W = np.array(rots, dtype=np.int32)
    Rxyz = np.array([L @ w @ Linv for w in W])
    return W, Rxyz
