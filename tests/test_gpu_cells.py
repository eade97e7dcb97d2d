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
