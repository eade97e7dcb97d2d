"""Host-side interface of the B200 path, mirroring SPRING's kappa.x procedures.

Each method of :class:`Context` wraps one C-ABI entry point of
``libspring_b200.so`` and names the reference procedure it replaces.  Arrays
are numpy arrays whose memory is the reference's Fortran array (C-order with
the Fortran axes reversed), e.g. ``Allq1q2(4,Nq)`` is returned as shape
``(Nq, 4)``.  Indices crossing the boundary are 1-based like the reference's.
Errors raise :class:`SpringError` with the library's message.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import _lib as L


class SpringError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"spring error {code}: {msg}")
        self.code = code


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ct.c_void_p)


def _c(a, dtype):
    return np.ascontiguousarray(a, dtype=dtype)


class Context:
    """One ``spring_ctx``: a crystal, a q-mesh and a list of temperatures on one GPU."""

    def __init__(self, nbasis: int, mesh, n_temps: int = 1, device: int = -1):
        self._lib = L.load()
        d = L.spring_dims()
        d.nbasis = int(nbasis)
        for k in range(3):
            d.mesh[k] = int(mesh[k])
        d.n_temps = int(n_temps)
        d.device = int(device)
        h = ct.c_void_p()
        rc = self._lib.spring_ctx_create(ct.byref(h), ct.byref(d))
        if rc != 0:
            raise SpringError(rc, "spring_ctx_create failed")
        self._h = h
        self.nbasis = int(nbasis)
        self.ndof = 3 * self.nbasis
        self.mesh = tuple(int(m) for m in mesh)
        self.nq = int(np.prod(self.mesh))
        self.n_temps = int(n_temps)
        self.nq0 = None

    # -- plumbing
    def _call(self, name, *args):
        rc = getattr(self._lib, name)(self._h, *args)
        if rc != 0:
            msg = self._lib.spring_last_error(self._h)
            raise SpringError(rc, (msg or b"").decode())

    def close(self):
        if getattr(self, "_h", None):
            self._lib.spring_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_stream(self, stream_ptr: int | None):
        self._call("spring_set_stream", ct.c_void_p(stream_ptr) if stream_ptr else None)

    def synchronize(self):
        self._call("spring_synchronize")

    def kernel_launches(self) -> int:
        n = ct.c_longlong()
        self._call("spring_kernel_launches", ct.byref(n))
        return int(n.value)

    def inject_fault(self, kind: int, n: int):
        self._call("spring_debug_inject_fault", int(kind), int(n))

    def set_option(self, option: int, value: int):
        self._call("spring_set_option", int(option), int(value))

    def set_precision(self, precision):
        """"fp64" (default), "bf16" or "bf16x3": arithmetic of the Gaussian V3 and V4 contractions."""
        code = {"fp64": L.SPRING_FP64, "bf16": L.SPRING_BF16, "bf16x3": L.SPRING_BF16X3}[precision]
        self._call("spring_set_precision", code)
        self._precision = precision

    @property
    def precision(self) -> str:
        """The arithmetic last set with set_precision ("fp64" until then)."""
        return getattr(self, "_precision", "fp64")

    # -- surrogate network (no counterpart in the reference)
    def mlp_init(self, seed: int = 0):
        self._call("spring_mlp_init", int(seed))

    def mlp_params(self):
        p = np.zeros(L.SPRING_MLP_PARAMS, np.float32)
        self._call("spring_mlp_get_params", _ptr(p))
        return p

    def mlp_set_params(self, p):
        self._call("spring_mlp_set_params", _ptr(_c(p, np.float32)))

    def mlp_loss_grad(self, X, y):
        X = _c(X, np.float32)
        y = _c(y, np.float32)
        loss = np.zeros(1, np.float32)
        g = np.zeros(L.SPRING_MLP_PARAMS, np.float32)
        self._call("spring_mlp_loss_grad", int(len(y)), _ptr(X), _ptr(y), _ptr(loss), _ptr(g))
        return float(loss[0]), g

    def mlp_train(self, X, y, epochs=100, batch=256, lr=1e-3, seed=0):
        X = _c(X, np.float32)
        y = _c(y, np.float32)
        hist = np.zeros(max(int(epochs), 1), np.float32)
        self._call("spring_mlp_train", int(len(y)), _ptr(X), _ptr(y), int(epochs), int(batch), float(lr), int(seed),
                   _ptr(hist))
        return hist[: int(epochs)]

    def mlp_predict(self, X, bf16=False):
        X = _c(X, np.float32)
        y = np.zeros(X.shape[0], np.float32)
        self._call("spring_mlp_predict", int(X.shape[0]), _ptr(X), _ptr(y), int(bool(bf16)))
        return y

    def use_generic_v3(self, on: bool = True):
        """Force the any-cell V3 kernel instead of the two-atom specialisation."""
        self.set_option(1, int(bool(on)))

    def set_profiling(self, on: bool):
        self._call("spring_set_profiling", int(bool(on)))

    def kernel_time(self, prefix: str):
        """(device ms, launches) of the recorded launches whose kernel name starts with ``prefix``."""
        ms = ct.c_double()
        n = ct.c_longlong()
        self._call("spring_kernel_time", prefix.encode(), ct.byref(ms), ct.byref(n))
        return float(ms.value), int(n.value)

    def tc_stats(self):
        """(tiles, pairs) of the last tensor-core linewidth pass: the pairs with a mode triple inside
        the delta window, cut into 16-pair tiles."""
        nt, npr = ct.c_int(), ct.c_int()
        self._call("spring_tc_stats", ct.byref(nt), ct.byref(npr))
        return int(nt.value), int(npr.value)

    def prepare3(self):
        self._call("spring_prepare3")

    # -- cell%init_data / FC readers
    def set_crystal(self, latvec, mass):
        lat = _c(np.asarray(latvec).T, np.float64)  # Fortran latvec(3,3): columns are vectors
        self._call("spring_set_crystal", _ptr(lat), _ptr(_c(mass, np.float64)))

    def set_dipole(self, basis_frac, eps, zstar, rmesh, decide=True, prec_ew=1e-6, lmb=0.8, gmesh=None,
                   sup_cell=(5, 5, 5)):
        """The dipole-dipole term (Force_dd): ``basis_frac`` (Nb, 3) fractional positions, ``eps`` the
        3x3 dielectric tensor with ``eps[i, j]`` = dielec(i, j), ``zstar`` (Nb, 3, 3) with
        ``zstar[mu][i, j]`` = BornZ(i, j, mu).  ``eps=None`` switches it off.  Set before the phonons
        are computed.  Returns (Lmb, Gmesh, number of R points, number of G points)."""
        if eps is None:
            self._call("spring_set_dipole", None, None, None, 0, 0.0, 0.0, None, None, None)
            return None
        bf = _c(basis_frac, np.float64)
        ep = _c(np.asarray(eps, np.float64).T, np.float64)               # Fortran order of dielec(3,3)
        zs = _c(np.asarray(zstar, np.float64).transpose(0, 2, 1), np.float64)  # BornZ(3,3,Nb)
        gm = _c(gmesh if gmesh is not None else (1, 1, 1), np.int32)
        self._call("spring_set_dipole", _ptr(bf), _ptr(ep), _ptr(zs), int(bool(decide)), float(prec_ew),
                   float(lmb), _ptr(gm), _ptr(_c(rmesh, np.int32)), _ptr(_c(sup_cell, np.int32)))
        on, lm, nr, ng = ct.c_int(), ct.c_double(), ct.c_int(), ct.c_int()
        g = np.zeros(3, np.int32)
        self._call("spring_get_dipole", ct.byref(on), ct.byref(lm), _ptr(g), ct.byref(nr), ct.byref(ng))
        return float(lm.value), tuple(int(x) for x in g), int(nr.value), int(ng.value)

    def set_point_defect(self, qmesh_pd, atm_num, atm_indx, fc2, mass_def, rho_def=1e-6, mat_inv_full=True,
                         optc_therm=True, phonons=None):
        """Point-defect scattering: the perturbed FC2 (same layout as :meth:`set_fc2`), the defect masses
        per basis atom, the defect density (A^-3) and the Green's-function mesh.  ``qmesh_pd=None``
        switches it off."""
        if qmesh_pd is None:
            self._call("spring_set_point_defect", None, 0, None, None, None, None, 0.0, 0, 0)
            return
        na = int(np.asarray(atm_indx).shape[1])
        self._call("spring_set_point_defect", _ptr(_c(qmesh_pd, np.int32)), na, _ptr(_c(atm_num, np.int32)),
                   _ptr(_c(atm_indx, np.int32)), _ptr(_c(fc2, np.float64)), _ptr(_c(mass_def, np.float64)),
                   float(rho_def), int(bool(mat_inv_full)), int(bool(optc_therm)))
        if phonons is not None:   # host phonons of the defect mesh (dict with evec, omega) instead of the device's
            self.set_phonons(2, None, phonons)

    def linewidth_pd(self, i0_first: int = 1, n_q0: int | None = None, add: bool = False):
        """Point-defect scattering rates (n_q0, Ndof); with add, 0.5 x rate joins LW_Allq0."""
        n_q0 = self.nq0 - i0_first + 1 if n_q0 is None else n_q0
        out = np.zeros((n_q0, self.ndof))
        self._call("spring_linewidth_pd", int(i0_first), int(n_q0), _ptr(out), int(bool(add)))
        return out

    def set_fc2(self, atm_num, atm_indx, fc2):
        na = int(np.asarray(atm_indx).shape[1])
        self._call("spring_set_fc2", na, _ptr(_c(atm_num, np.int32)), _ptr(_c(atm_indx, np.int32)),
                   _ptr(_c(fc2, np.float64)))

    def set_fc3(self, atm_num, atm_indx, fc3):
        na = int(np.asarray(atm_indx).shape[1])
        self._call("spring_set_fc3", na, _ptr(_c(atm_num, np.int32)), _ptr(_c(atm_indx, np.int32)),
                   _ptr(_c(fc3, np.float64)))

    def set_fc4(self, atm_num, atm_indx, fc4):
        na = int(np.asarray(atm_indx).shape[1])
        self._call("spring_set_fc4", na, _ptr(_c(atm_num, np.int32)), _ptr(_c(atm_indx, np.int32)),
                   _ptr(_c(fc4, np.float64)))

    # -- q_tetrahedron
    def make_mesh(self, shift=(0, 0, 0), zero_centered=True, want=True):
        sh = _c(shift, np.int32)
        if not want:
            self._call("spring_make_mesh", _ptr(sh), int(zero_centered), None, None, None)
            return None
        qi = np.zeros((self.nq, 3), np.int32)
        qf = np.zeros((self.nq, 3), np.float64)
        tet = np.zeros((6 * self.nq, 4), np.int32)
        self._call("spring_make_mesh", _ptr(sh), int(zero_centered), _ptr(qi), _ptr(qf), _ptr(tet))
        return qi, qf, tet

    def find_irr_q(self, rotations, time_rev=0):
        rot = _c(rotations, np.int32)  # (nrot, 3, 3) row-major W
        nq0 = ct.c_int()
        irr = np.zeros((self.nq, 3), np.int32)
        pos = np.zeros(self.nq, np.int32)
        mult = np.zeros(self.nq, np.int32)
        self._call("spring_find_irr_q", int(rot.shape[0]), _ptr(rot), int(time_rev), ct.byref(nq0), _ptr(irr),
                   _ptr(pos), _ptr(mult))
        self.nq0 = int(nq0.value)
        return dict(irr_q_pnt_int=irr[: self.nq0].copy(), pos=pos, multiplicity=mult[: self.nq0].copy())

    # -- Phon
    def compute_phonons(self, temps, freq_cut=2.56789e-5):
        self._call("spring_compute_phonons", _ptr(_c(temps, np.float64)), float(freq_cut))

    def set_phonons(self, which: int, temps, ph: dict):
        """which 0: grid, 1: irreducible set, 2: the point-defect mesh (evec and omega only)."""
        if which == 2:
            self._call("spring_set_phonons", 2, None, _ptr(_c(ph["evec"], np.complex128)),
                       _ptr(_c(ph["omega"], np.float64)), None, None, None)
            return
        self._call("spring_set_phonons", int(which), _ptr(_c(temps, np.float64)), _ptr(_c(ph["evec"], np.complex128)),
                   _ptr(_c(ph["omega"], np.float64)), _ptr(_c(ph["onebyomega"], np.float64)),
                   _ptr(_c(ph["nbe"], np.float64)), _ptr(_c(ph["grp_vel"], np.float64)))

    def get_phonons(self, which: int) -> dict:
        n = self.nq if which == 0 else self.nq0
        nd = self.ndof
        out = dict(evec=np.zeros((n, nd, nd), np.complex128), omega=np.zeros((n, nd)), onebyomega=np.zeros((n, nd)),
                   nbe=np.zeros((self.n_temps, n, nd)), grp_vel=np.zeros((n, nd, 3)))
        self._call("spring_get_phonons", int(which), _ptr(out["evec"]), _ptr(out["omega"]), _ptr(out["onebyomega"]),
                   _ptr(out["nbe"]), _ptr(out["grp_vel"]))
        return out

    # -- MomentumConsrv3rd
    def enumerate3(self, i0: int):
        A = np.zeros((self.nq, 4), np.int32)
        Pm = np.zeros((self.nq, 2), np.int32)
        cnt = np.zeros(2, np.int32)
        self._call("spring_enumerate3", int(i0), _ptr(A), _ptr(Pm), _ptr(cnt))
        return A, Pm[: cnt[0]].copy(), (int(cnt[0]), int(cnt[1]))

    # -- MomentumConsrv4th
    def count4(self, i0: int):
        """(q1q2q3_count, total_count) of q0 = i0, without copying the lists back."""
        cnt = np.zeros(2, np.int64)
        self._call("spring_enumerate4", int(i0), None, None, 0, _ptr(cnt))
        return int(cnt[0]), int(cnt[1])

    def enumerate4(self, i0: int, cap=None):
        """Allq1q2q3 [q1][q2][3], q1q2q3_permuted [quartet][3] (1-based) and (count, total_count)."""
        A = np.zeros((self.nq, self.nq, 3), np.int32)
        cap = self.nq * self.nq if cap is None else int(cap)
        Pm = np.zeros((max(cap, 1), 3), np.int32)
        cnt = np.zeros(2, np.int64)
        self._call("spring_enumerate4", int(i0), _ptr(A), _ptr(Pm), cap, _ptr(cnt))
        return A, Pm[: cnt[0]].copy(), (int(cnt[0]), int(cnt[1]))

    # -- ScatterProbAllq1
    def scatter_w3(self, i0: int):
        nd = self.ndof
        out = np.zeros((self.nq, nd, nd, nd))
        self._call("spring_scatter_w3", int(i0), _ptr(out))
        return out

    # -- linewidths
    def linewidth3(self, i0_first: int, n_q0: int, delta: str = "gauss", sigma: float = 0.3767, pol3=None,
                   want=True, out=None):
        """``want=False``: results stay on the device; ``out``: a caller-owned (nT, n_q0, Ndof) float64
        array (e.g. pinned) that receives the linewidths, without the phase space."""
        mode = L.SPRING_DELTA_GAUSS if delta == "gauss" else L.SPRING_DELTA_TETRA
        pol = None if pol3 is None else _c(pol3, np.int32)
        if out is not None:
            assert out.dtype == np.float64 and out.flags.c_contiguous and out.shape == (self.n_temps, n_q0, self.ndof)
            self._call("spring_linewidth3", int(i0_first), int(n_q0), mode, float(sigma), _ptr(pol), _ptr(out), None)
            return out
        if not want:
            self._call("spring_linewidth3", int(i0_first), int(n_q0), mode, float(sigma), _ptr(pol), None, None)
            return None
        lw = np.zeros((self.n_temps, n_q0, self.ndof))
        p3 = np.zeros((n_q0, self.ndof))
        self._call("spring_linewidth3", int(i0_first), int(n_q0), mode, float(sigma), _ptr(pol), _ptr(lw), _ptr(p3))
        return lw, p3

    def linewidth_iso(self, i0_first: int, n_q0: int, g2, delta: str = "gauss", sigma: float = 0.3767, want=True):
        mode = L.SPRING_DELTA_GAUSS if delta == "gauss" else L.SPRING_DELTA_TETRA
        g = _c(g2, np.float64)
        if not want:
            self._call("spring_linewidth_iso", int(i0_first), int(n_q0), mode, float(sigma), _ptr(g), None)
            return None
        rate = np.zeros((self.n_temps, n_q0, self.ndof))
        self._call("spring_linewidth_iso", int(i0_first), int(n_q0), mode, float(sigma), _ptr(g), _ptr(rate))
        return rate

    def linewidth4(self, i0_first: int, n_q0: int, delta: str = "tetra", sigma: float = 0.3767, pol4=None,
                   want=True):
        """Four-phonon scattering rate (nT, n_q0, Ndof); 0.5 x rate joins the resident linewidths."""
        mode = L.SPRING_DELTA_GAUSS if delta == "gauss" else L.SPRING_DELTA_TETRA
        pol = None if pol4 is None else _c(pol4, np.int32)
        if not want:
            self._call("spring_linewidth4", int(i0_first), int(n_q0), mode, float(sigma), _ptr(pol), None)
            return None
        rate = np.zeros((self.n_temps, n_q0, self.ndof))
        self._call("spring_linewidth4", int(i0_first), int(n_q0), mode, float(sigma), _ptr(pol), _ptr(rate))
        return rate

    def linewidth4_modes(self, i0_first: int, s0_mask, sigma: float = 0.3767):
        """Gaussian four-phonon rates (nT, n_q0, Ndof) of the selected branches only (bit s of
        s0_mask[k] selects branch s of q0 = i0_first + k), zero elsewhere; LW_Allq0 untouched."""
        m = _c(s0_mask, np.int32)
        n = int(m.shape[0])
        rate = np.zeros((self.n_temps, n, self.ndof))
        self._call("spring_linewidth4_modes", int(i0_first), n, float(sigma), _ptr(m), _ptr(rate))
        return rate

    # -- LineWidth.x path mode
    def path_qpoints(self, q_high_sym):
        """q_points_highsymm: (qpoints (n, 3) Cartesian, dist (n,), zero_centered (n,) bool)."""
        qhs = _c(q_high_sym, np.float64)  # (n_nodes, 4): fractional node, point count
        n_rows = ct.c_int()
        self._call("spring_path_qpoints", int(qhs.shape[0]), _ptr(qhs), ct.byref(n_rows), None, None, None)
        n = int(n_rows.value)
        q = np.zeros((max(n, 1), 3))
        d = np.zeros(max(n, 1))
        z = np.zeros(max(n, 1), np.int32)
        self._call("spring_path_qpoints", int(qhs.shape[0]), _ptr(qhs), ct.byref(n_rows), _ptr(q), _ptr(d), _ptr(z))
        return q[:n], d[:n], z[:n].astype(bool)

    def linewidth_path(self, q0, zero_centered, delta: str = "tetra", sigma: float = 0.3767):
        """Linewidths (nT, n_q0, Ndof) and frequencies (n_q0, Ndof) at off-grid q0 points."""
        q = _c(q0, np.float64).reshape(-1, 3)
        z = _c(zero_centered, np.int32)
        mode = L.SPRING_DELTA_GAUSS if delta == "gauss" else L.SPRING_DELTA_TETRA
        lw = np.zeros((self.n_temps, q.shape[0], self.ndof))
        om = np.zeros((q.shape[0], self.ndof))
        self._call("spring_linewidth_path", int(q.shape[0]), _ptr(q), _ptr(z), mode, float(sigma), _ptr(lw), _ptr(om))
        return lw, om

    def reset_linewidths(self):
        self._call("spring_reset_linewidths")

    def get_linewidths(self):
        out = np.zeros((self.n_temps, self.nq0, self.ndof))
        self._call("spring_get_linewidths", _ptr(out))
        return out

    def set_linewidths(self, lw):
        self._call("spring_set_linewidths", _ptr(_c(lw, np.float64)))

    # -- kappa_noIter(_symm)
    def kappa_rta(self, Rxyz=None, symm=True, s_range=None, mode=False, want=True, out=None):
        R = None
        nsym = 0
        if symm:
            R = _c(np.transpose(np.asarray(Rxyz), (0, 2, 1)), np.float64)  # Rxyz(3,3,Nsym) column-major
            nsym = R.shape[0]
        sr = None if s_range is None else _c(s_range, np.int32)
        if not want:
            self._call("spring_kappa_rta", int(bool(symm)), nsym, _ptr(R), _ptr(sr), None, None)
            return None
        kap = np.zeros((self.n_temps, 9)) if out is None else out
        mk = np.zeros((self.n_temps, self.ndof, 9)) if mode else None
        self._call("spring_kappa_rta", int(bool(symm)), nsym, _ptr(R), _ptr(sr), _ptr(kap), _ptr(mk))
        return (kap, mk) if mode else kap


    # -- kappa_iter.x
    def kappa_iter(self, eps_k: float = 1e-6, max_iter: int = 1000):
        """Iterative kappa per temperature: dict(kappa (nT,9), kappa_rta (nT,9), iters (nT,))."""
        kap = np.zeros((self.n_temps, 9))
        k0 = np.zeros((self.n_temps, 9))
        it = np.zeros(self.n_temps, np.int32)
        self._call("spring_kappa_iter", float(eps_k), int(max_iter), _ptr(kap), _ptr(k0), _ptr(it))
        return dict(kappa=kap, kappa_rta=k0, iters=it)

    def kappa_iter_gauss(self, sigma: float, eps_k: float = 1e-6, max_iter: int = 1000):
        """Iterative kappa with Gaussian delta weights of width sigma (THz): dict(kappa (nT,9),
        kappa_rta (nT,9), iters (nT,), entries, pairs)."""
        kap = np.zeros((self.n_temps, 9))
        k0 = np.zeros((self.n_temps, 9))
        it = np.zeros(self.n_temps, np.int32)
        st = np.zeros(2)
        self._call("spring_kappa_iter_gauss", float(sigma), float(eps_k), int(max_iter), _ptr(kap), _ptr(k0),
                   _ptr(it), _ptr(st))
        return dict(kappa=kap, kappa_rta=k0, iters=it, entries=int(st[0]), pairs=int(st[1]))


def from_crystal(cr, mesh, temps, phonons="device", W=None, Rxyz=None, with_fc3=True, with_fc4=False,
                 dipole=None):
    """A ready context for a :class:`spring_b200.synthetic.Crystal`.

    ``phonons="device"`` computes them with the device eigensolver; a dict
    ``{"grid": ph, "irr": ph}`` loads host-computed ones instead.  ``dipole``: keyword
    arguments of :meth:`Context.set_dipole` (rmesh, decide, prec_ew, ...) to add the
    dipole-dipole term with the crystal's Born charges and dielectric tensor.
    Returns ``(ctx, info)`` where ``info`` holds the mesh and irreducible set.
    """
    from . import synthetic as S
    temps = np.atleast_1d(np.asarray(temps, np.float64))
    ctx = Context(cr.nbasis, mesh, len(temps))
    ctx.set_crystal(cr.latvec, cr.mass)
    ctx.set_fc2(cr.fc2_atm_num, cr.fc2_atm_indx, cr.fc2)
    if with_fc3:
        ctx.set_fc3(cr.fc3_atm_num, cr.fc3_atm_indx, cr.fc3)
    if with_fc4:
        ctx.set_fc4(cr.fc4_atm_num, cr.fc4_atm_indx, cr.fc4)
    ew = ctx.set_dipole(cr.basis_frac, cr.eps, cr.zstar, **dipole) if dipole is not None else None
    qi, qf, tet = ctx.make_mesh()
    if W is None:
        W, Rxyz = S.point_group(cr)
    irr = ctx.find_irr_q(W)
    if isinstance(phonons, dict):
        ctx.set_phonons(0, temps, phonons["grid"])
        ctx.set_phonons(1, temps, phonons["irr"])
    else:
        ctx.compute_phonons(temps)
    info = dict(q_pnt_int=qi, q_pnt=qf, tetra=tet, W=W, Rxyz=Rxyz, temps=temps, ewald=ew, **irr)
    return ctx, info


class Batch:
    """A ``spring_batch``: Gaussian three-phonon linewidth requests on several contexts (cells,
    meshes, temperature sets) run as one persistent, graph-captured launch."""

    def __init__(self):
        self._lib = L.load()
        h = ct.c_void_p()
        rc = self._lib.spring_batch_create(ct.byref(h))
        if rc != 0:
            raise SpringError(rc, "spring_batch_create failed")
        self._h = h
        self._reqs = []
        self._paths = []

    def _call(self, name, *args):
        rc = getattr(self._lib, name)(self._h, *args)
        if rc != 0:
            msg = self._lib.spring_batch_last_error(self._h)
            raise SpringError(rc, (msg or b"").decode())

    def add_linewidth3(self, ctx: Context, i0_first: int, n_q0: int, sigma: float, pol=None) -> int:
        """Queue spring_linewidth3(ctx, i0_first, n_q0, Gaussian, sigma, pol); returns its index."""
        idx = ct.c_int()
        polp = None if pol is None else np.ascontiguousarray(pol, dtype=np.int32)
        self._call("spring_batch_add_linewidth3", ctx._h, int(i0_first), int(n_q0), float(sigma), _ptr(polp),
                   ct.byref(idx))
        self._reqs.append((ctx, int(n_q0)))
        return idx.value

    def add_path(self, ctx: Context, q0, zero_centered, sigma: float) -> int:
        """Queue Gaussian linewidths at off-grid points q0 (n, 3) of ``ctx`` (the path mode of
        spring_linewidth_path); they run inside the batch's graph.  Returns the path request's index."""
        q = _c(q0, np.float64).reshape(-1, 3)
        z = _c(zero_centered, np.int32)
        idx = ct.c_int()
        self._call("spring_batch_add_path", ctx._h, int(q.shape[0]), _ptr(q), _ptr(z), float(sigma), ct.byref(idx))
        self._paths.append((ctx, int(q.shape[0]), q, z))
        return idx.value

    def path_result(self, index: int):
        """(lw[T][n][Ndof], omega[n][Ndof]) of path request ``index`` after the last run."""
        if not 0 <= index < len(self._paths):
            self._call("spring_batch_path_result", int(index), None, None)  # raises: no such request
        ctx, n, _, _ = self._paths[index]
        lw = np.zeros((ctx.n_temps, n, ctx.ndof))
        om = np.zeros((n, ctx.ndof))
        self._call("spring_batch_path_result", int(index), _ptr(lw), _ptr(om))
        return lw, om

    def set_config(self, two_atom=1, ctas_per_sm=0, s0_block=0, chunk=1):
        """two_atom: run two-atom cells in the specialised 8-pair layout; ctas_per_sm (0: as many as
        fit); s0_block for Ndof > 12 (0: 6); chunk: work items per scheduler step."""
        cfg = np.array([two_atom, ctas_per_sm, s0_block, chunk], dtype=np.int32)
        self._call("spring_batch_set_config", _ptr(cfg))

    def config(self):
        cfg = np.zeros(4, dtype=np.int32)
        self._call("spring_batch_get_config", _ptr(cfg))
        return tuple(int(x) for x in cfg)

    def tune(self):
        """Autotune the launch configuration; returns (config, best ms, configurations tried)."""
        cfg = np.zeros(4, dtype=np.int32)
        ms = ct.c_double()
        n = ct.c_int()
        self._call("spring_batch_tune", _ptr(cfg), ct.byref(ms), ct.byref(n))
        return tuple(int(x) for x in cfg), ms.value, n.value

    def run(self):
        self._call("spring_batch_run")

    def result(self, index: int):
        """(lw[T][n_q0][Ndof], p3[n_q0][Ndof], ms of the last run) of request ``index``."""
        ctx, n_q0 = self._reqs[index]
        lw = np.zeros((ctx.n_temps, n_q0, ctx.ndof))
        p3 = np.zeros((n_q0, ctx.ndof))
        ms = ct.c_double()
        self._call("spring_batch_result", int(index), _ptr(lw), _ptr(p3), ct.byref(ms))
        return lw, p3, ms.value

    def close(self):
        if getattr(self, "_h", None):
            self._lib.spring_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
