"""Cells and temperature counts beyond the two-atom, three-temperature case: the 8-atom cubic
rocksalt cell (24 branches, s0 blocks in the V3 kernel) and nine temperatures (100-900 K) in one
call, on the FP64 and the tensor-core paths, against the CPU oracle.  (Kappa is not compared at 5^3:
a few modes there have no scattering partner inside the Gaussian and their lifetime diverges.)"""
import numpy as np
import pytest

from oracle import driver as D
from spring_b200 import synthetic as S
from spring_b200.api import from_crystal

pytestmark = pytest.mark.gpu

TEMPS9 = [100.0 * k for k in range(1, 10)]


@pytest.mark.parametrize("delta", ["gauss", "tetra"])
def test_eight_atom_cell(delta):
    cr = S.build("rocksalt8")
    N = 2
    st = D.Setup(cr, (N, N, N), [300.0, 700.0])
    ctx, info = from_crystal(cr, (N, N, N), st.temps, phonons={"grid": st.ph, "irr": st.ph0})
    assert ctx.ndof == 24
    ctx.reset_linewidths()
    lw, _ = ctx.linewidth3(1, ctx.nq0, delta, 0.8)
    for i0 in range(st.nq0):
        for it in range(2):
            ref = D.linewidth3_q0(st, i0, delta, 0.8, it=it)["lw"]
            scale = np.abs(ref).max()
            np.testing.assert_allclose(lw[it, i0], ref, rtol=1e-8, atol=1e-11 * scale)
    ctx.close()


def test_nine_temperatures_fp64_and_tensor_cores():
    cr = S.build("rocksalt2")
    N = 5
    st = D.Setup(cr, (N, N, N), TEMPS9)
    ctx, info = from_crystal(cr, (N, N, N), TEMPS9, phonons={"grid": st.ph, "irr": st.ph0})
    ctx.reset_linewidths()
    lw64, p364 = ctx.linewidth3(1, ctx.nq0, "gauss", 1.0)
    for i0 in (0, st.nq0 // 2, st.nq0 - 1):
        for it in (0, 4, 8):
            ref = D.linewidth3_q0(st, i0, "gauss", 1.0, it=it)["lw"]
            np.testing.assert_allclose(lw64[it, i0], ref, rtol=1e-9, atol=1e-12 * np.abs(ref).max())
    ctx.set_precision("bf16x3")
    ctx.reset_linewidths()
    lw, p3 = ctx.linewidth3(1, ctx.nq0, "gauss", 1.0)
    ctx.set_precision("fp64")
    for it in range(9):
        big = lw64[it] > 1e-3 * lw64[it].max()
        assert (np.abs(lw[it][big] - lw64[it][big]) / lw64[it][big]).max() < 1e-4
    np.testing.assert_allclose(p3, p364, rtol=1e-10, atol=1e-12 * np.abs(p364).max())
    ctx.close()


@pytest.mark.parametrize("N", [2, 3])
def test_eight_atom_device_phonons_vs_lapack(N):
    """The any-cell device eigensolver (k_phonons, Ndof 24: one CTA per q-point, cyclic complex
    Jacobi) against LAPACK zheevd through the oracle: eigenvalues, occupations, eigen-projectors of
    non-degenerate modes and their group velocities, on the grid and the irreducible points."""
    cr = S.build("rocksalt8")
    st = D.Setup(cr, (N, N, N), [300.0])
    ctx, _ = from_crystal(cr, (N, N, N), st.temps, phonons="device")
    assert ctx.ndof == 24
    for which, ref in ((0, st.ph), (1, st.ph0)):
        ph = ctx.get_phonons(which)
        lam, lam_ref = np.sign(ph["omega"]) * ph["omega"] ** 2, np.sign(ref["omega"]) * ref["omega"] ** 2
        np.testing.assert_allclose(lam, lam_ref, rtol=1e-10, atol=1e-9 * np.abs(lam_ref).max())
        np.testing.assert_allclose(ph["nbe"], ref["nbe"], rtol=1e-8, atol=1e-12)
        nd = ctx.ndof
        for q in range(ref["omega"].shape[0]):
            w = ref["omega"][q]
            for s in range(nd):
                gap = np.min(np.abs(np.delete(w, s) - w[s]))
                if gap < 1e-3 * max(1.0, abs(w[s])) or abs(w[s]) < 1e-3:
                    continue
                e, f = ph["evec"][q, s], ref["evec"][q, s]
                np.testing.assert_allclose(np.outer(e, e.conj()), np.outer(f, f.conj()), atol=1e-9)
                np.testing.assert_allclose(ph["grp_vel"][q, s], ref["grp_vel"][q, s], rtol=1e-7, atol=1e-6)
        # (near-)degenerate subspaces: the projector onto each cluster of close frequencies (the
        # modes skipped above) is gauge-free
        for q in range(ref["omega"].shape[0]):
            w = ref["omega"][q]
            s = 0
            while s < nd:
                t = s + 1
                while t < nd and (abs(w[t] - w[t - 1]) < 1e-3 * max(1.0, abs(w[t])) or abs(w[t]) < 1e-3):
                    t += 1
                E, F = ph["evec"][q, s:t], ref["evec"][q, s:t]
                np.testing.assert_allclose(E.T @ E.conj(), F.T @ F.conj(), atol=1e-8)
                s = t
    ctx.close()
