"""Iterative BTE (kappa_iter.x) on the GPU against the CPU oracle."""
import numpy as np
import pytest

from oracle import driver as D
from spring_b200 import synthetic as S
from spring_b200.api import from_crystal

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N", [4, 5])
def test_kappa_iter_matches_oracle(N):
    cr = S.build("rocksalt2")
    st = D.Setup(cr, (N, N, N), [300.0, 700.0])
    ctx, _ = from_crystal(cr, (N, N, N), st.temps, phonons={"grid": st.ph, "irr": st.ph0})
    out = ctx.kappa_iter(eps_k=1e-6)
    for it in range(2):
        ref = D.bte_iter(st, it=it, eps_k=1e-6)
        np.testing.assert_allclose(out["kappa_rta"][it], ref["kappa_rta"], rtol=1e-9,
                                   atol=1e-12 * np.abs(ref["kappa_rta"]).max())
        assert abs(int(out["iters"][it]) - ref["iters"]) <= 1
        np.testing.assert_allclose(out["kappa"][it], ref["kappa"], rtol=1e-6, atol=1e-9 * np.abs(ref["kappa"]).max())
    ctx.close()


@pytest.mark.parametrize("N,sigma", [(5, 1.5), (6, 0.8)])
def test_kappa_iter_gauss_tensor_core_operator(N, sigma):
    """On a BF16x3 context the operator entries come from the tensor-core pass: the same entries
    (the window and the cuts are the FP64 ones, only |Phi|^2 is compensated BF16), kappa and the RTA
    start within 1e-5 of the FP64 operator's; switching back to FP64 rebuilds the FP64 operator."""
    cr = S.build("rocksalt2")
    st = D.Setup(cr, (N, N, N), [300.0, 700.0])
    ctx, _ = from_crystal(cr, (N, N, N), st.temps, phonons={"grid": st.ph, "irr": st.ph0})
    ref = ctx.kappa_iter_gauss(sigma, eps_k=1e-6)
    ctx.set_precision("bf16x3")
    out = ctx.kappa_iter_gauss(sigma, eps_k=1e-6)
    assert out["entries"] == ref["entries"] and out["pairs"] == ref["pairs"]
    for it in range(2):
        for key in ("kappa_rta", "kappa"):
            scale = np.abs(ref[key][it]).max()
            # within 1e-5 of the tensor's largest component (the small off-diagonal terms included)
            np.testing.assert_allclose(out[key][it], ref[key][it], rtol=1e-5, atol=1e-5 * scale)
        assert abs(int(out["iters"][it]) - int(ref["iters"][it])) <= 1
    ctx.set_precision("fp64")
    back = ctx.kappa_iter_gauss(sigma, eps_k=1e-6)
    np.testing.assert_allclose(back["kappa"], ref["kappa"], rtol=1e-12, atol=0.0)
    ctx.close()


def test_kappa_iter_rta_equals_kappa_x_full_grid():
    """Iteration 0 of the BTE is kappa.x's RTA on the full grid (identity symmetry)."""
    cr = S.build("rocksalt2")
    N = 4
    W = np.eye(3, dtype=np.int32)[None]
    st = D.Setup(cr, (N, N, N), [300.0], W=W, Rxyz=np.eye(3)[None])
    ctx, info = from_crystal(cr, (N, N, N), st.temps, phonons={"grid": st.ph, "irr": st.ph0}, W=W,
                             Rxyz=np.eye(3)[None])
    ctx.linewidth3(1, ctx.nq0, delta="tetra", want=False)
    k_rta = ctx.kappa_rta(symm=False)[0]
    out = ctx.kappa_iter(eps_k=1e-6)
    np.testing.assert_allclose(out["kappa_rta"][0], k_rta, rtol=1e-9, atol=1e-12 * np.abs(k_rta).max())
    ctx.close()


@pytest.mark.parametrize("N,sigma", [(4, 1.5), (5, 1.5), (6, 0.8)])
def test_kappa_iter_gauss_matches_oracle(N, sigma):
    """The Gaussian operator form of the iteration: 1/tau, the RTA start and the converged kappa
    against the oracle's per-channel sums over the full W3 grids (two temperatures)."""
    cr = S.build("rocksalt2")
    st = D.Setup(cr, (N, N, N), [300.0, 700.0])
    ctx, _ = from_crystal(cr, (N, N, N), st.temps, phonons={"grid": st.ph, "irr": st.ph0})
    out = ctx.kappa_iter_gauss(sigma, eps_k=1e-6)
    assert out["entries"] > 0 and out["pairs"] > 0
    again = ctx.kappa_iter_gauss(sigma, eps_k=1e-6)   # the kept operator gives the same answer
    np.testing.assert_array_equal(again["kappa"], out["kappa"])
    for it in range(2):
        ref = D.bte_iter_gauss(st, sigma, it=it, eps_k=1e-6)
        np.testing.assert_allclose(out["kappa_rta"][it], ref["kappa_rta"], rtol=1e-9,
                                   atol=1e-12 * np.abs(ref["kappa_rta"]).max())
        assert abs(int(out["iters"][it]) - ref["iters"]) <= 1
        np.testing.assert_allclose(out["kappa"][it], ref["kappa"], rtol=1e-6, atol=1e-9 * np.abs(ref["kappa"]).max())
    ctx.close()

