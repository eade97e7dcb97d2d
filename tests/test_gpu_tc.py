"""Tensor-core (tcgen05) V3 in the fused Gaussian linewidth: BF16 and compensated BF16x3 against the
FP64 GPU path and the CPU oracle.  Tolerances are the accuracy targets of the mixed-precision path:
linewidths within 2 % and kappa within 1 % of FP64 (BF16), and 1e-4 / 1e-5 for the compensated form."""
import numpy as np
import pytest

from oracle import driver as D
from spring_b200 import synthetic as S
from spring_b200.api import from_crystal

pytestmark = pytest.mark.gpu

TEMPS = [100.0, 300.0, 700.0]
SIGMA = 0.3767


@pytest.fixture(scope="module", params=[8, 12])
def runs(request):
    cr = S.build("rocksalt2")
    N = request.param
    st = D.Setup(cr, (N, N, N), TEMPS)
    ctx, info = from_crystal(cr, (N, N, N), TEMPS, phonons={"grid": st.ph, "irr": st.ph0})
    out = {}
    for prec in ("fp64", "bf16x3", "bf16"):
        ctx.set_precision(prec)
        ctx.reset_linewidths()
        lw, p3 = ctx.linewidth3(1, ctx.nq0, "gauss", SIGMA)
        kap = ctx.kappa_rta(info["Rxyz"])
        out[prec] = (lw, p3, kap)
    ctx.set_precision("fp64")
    yield N, ctx, info, out, st
    ctx.close()


@pytest.mark.parametrize("prec,lw_tol,k_tol", [("bf16x3", 1e-4, 1e-5), ("bf16", 2e-2, 1e-2)])
def test_tc_linewidths_and_kappa_vs_fp64(runs, prec, lw_tol, k_tol):
    N, ctx, info, out, _ = runs
    lw64, p364, k64 = out["fp64"]
    lw, p3, k = out[prec]
    for it in range(len(TEMPS)):
        big = lw64[it] > 1e-3 * lw64[it].max()   # every mode whose linewidth is not negligible
        rel = np.abs(lw[it][big] - lw64[it][big]) / lw64[it][big]
        assert rel.max() < lw_tol, (prec, it, rel.max())
        diag = np.array([k64[it][0], k64[it][4], k64[it][8]])
        kd = np.array([k[it][0], k[it][4], k[it][8]])
        assert np.abs(kd / diag - 1).max() < k_tol, (prec, it, kd, diag)
    # the delta weights stay FP64: the phase space differs only by the exp cut (< 4e-18 of a peak)
    np.testing.assert_allclose(p3, p364, rtol=1e-10, atol=1e-12 * np.abs(p364).max())


def test_tc_matches_oracle_at_8(runs):
    N, ctx, info, out, st = runs
    if N != 8:
        pytest.skip("oracle comparison on the 8^3 mesh only")
    lw, _, _ = out["bf16x3"]
    for i0 in (0, 3, st.nq0 - 1):
        ref = D.linewidth3_q0(st, i0, "gauss", SIGMA, it=1)["lw"]
        big = ref > 1e-3 * ref.max()
        assert (np.abs(lw[1, i0][big] - ref[big]) / ref[big]).max() < 1e-4


def test_tc_pair_subset_and_repeat(runs):
    """A q0 block smaller than the whole set, called twice (tile cache reuse), equals the full run."""
    N, ctx, info, out, _ = runs
    lw_all, _, _ = out["bf16x3"]
    ctx.set_precision("bf16x3")
    for _ in range(2):
        ctx.reset_linewidths()
        lw, _ = ctx.linewidth3(2, 3, "gauss", SIGMA)
        np.testing.assert_allclose(lw, lw_all[:, 1:4], rtol=1e-12, atol=1e-15)
    ctx.set_precision("fp64")


def test_tc_pair_prescreen_follows_sigma_and_phonons(runs):
    """Pairs with no mode triple inside the delta window are left out of the tiles; the tiles are
    rebuilt when the Gaussian width or the phonons change.  The phase space (FP64 delta weights of
    every triple above the exp cut) shows a dropped pair at once, so it is compared at 1e-10."""
    N, ctx, info, out, st = runs
    if N != 8:
        pytest.skip("8^3 mesh only")

    def both(sigma):
        res = {}
        for prec in ("fp64", "bf16x3"):
            ctx.set_precision(prec)
            ctx.reset_linewidths()
            res[prec] = ctx.linewidth3(1, ctx.nq0, "gauss", sigma)
        ctx.set_precision("fp64")
        return res

    for sigma in (0.05, 1.5, SIGMA):  # narrow window (most pairs dropped), wide (few), default
        r = both(sigma)
        p64, p = r["fp64"][1], r["bf16x3"][1]
        np.testing.assert_allclose(p, p64, rtol=1e-10, atol=1e-12 * np.abs(p64).max())
        lw64, lw = r["fp64"][0], r["bf16x3"][0]
        big = lw64 > 1e-3 * lw64.max()
        assert (np.abs(lw[big] - lw64[big]) / lw64[big]).max() < 1e-4, sigma
    np.testing.assert_allclose(r["bf16x3"][0], out["bf16x3"][0], rtol=1e-12, atol=1e-15)
    # a window almost no pair reaches (possibly none: then nothing is launched); the FP64 path keeps
    # the Gaussian tails below exp(-40) of the peak that the tensor-core path drops, at most
    # 3 channels x weight 2 x exp(-40) / (sqrt(2 pi) sigma) per mode triple
    sig = 1e-7
    r = both(sig)
    cut = 6.0 * np.exp(-40.0) / (np.sqrt(2.0 * np.pi) * sig) * ctx.nq * 216
    np.testing.assert_allclose(r["bf16x3"][1], r["fp64"][1], rtol=1e-10, atol=cut)
    # new grid phonons (frequencies scaled by 1.05): the cached tiles must not be reused
    ph = {k: np.array(v, copy=True) for k, v in st.ph.items()}
    ph["omega"] = ph["omega"] * 1.05
    ph["onebyomega"] = ph["onebyomega"] / 1.05
    ctx.set_phonons(0, TEMPS, ph)
    try:
        r = both(SIGMA)
        p64, p = r["fp64"][1], r["bf16x3"][1]
        np.testing.assert_allclose(p, p64, rtol=1e-10, atol=1e-12 * np.abs(p64).max())
    finally:
        ctx.set_phonons(0, TEMPS, st.ph)


def test_tc_prescreen_counts_match_numpy(runs):
    """The pairs the tensor-core pass keeps (and their 16-pair tiles per q1) are exactly those a
    float32 restatement of the delta-window test keeps: |(|w1| - |w0 - w2|)| < R or |w0 + w2 - w1| < R
    for some mode triple, R = sqrt(40 / (0.5 / sigma^2)) * 1.0001 + 1e-3."""
    N, ctx, info, out, st = runs
    if N != 8:
        pytest.skip("8^3 mesh only")
    ctx.set_precision("bf16x3")
    ctx.reset_linewidths()
    ctx.linewidth3(1, ctx.nq0, "gauss", SIGMA)
    tiles, pairs = ctx.tc_stats()
    ctx.set_precision("fp64")
    os_ = 1.0 / SIGMA
    rf = np.float32(np.sqrt(40.0 / (0.5 * (os_ * os_))) * 1.0001 + 1e-3)
    om = st.ph["omega"].astype(np.float32)
    om0 = st.ph0["omega"].astype(np.float32)
    kept = 0
    by_q1 = np.zeros(st.nq, np.int64)
    for i0 in range(st.nq0):
        _, perm, cnt = D.momentum3(st.mesh, st.q_pnt_int, st.irr_int[i0])
        q1 = perm[: cnt[0], 0] - 1
        q2 = perm[: cnt[0], 1] - 1
        w0 = om0[i0][None, :, None, None]
        w1 = om[q1][:, None, :, None]
        w2 = om[q2][:, None, None, :]
        a = (np.abs(np.abs(w1) - np.abs(w0 - w2)) < rf) | (np.abs((w0 + w2) - w1) < rf)
        m = a.reshape(cnt[0], -1).any(1)
        kept += int(m.sum())
        np.add.at(by_q1, q1[m], 1)
    assert pairs == kept
    assert tiles == int(((by_q1 + 15) // 16).sum())


def test_tc_wait_timeout_returns_status_and_context_recovers(runs):
    """Every wait of one warp on another in the tensor-core kernel is bounded.  With a poll limit of 0
    each such wait runs out at once: the kernel drains the copies it issued, frees its tensor memory
    and returns, the call fails with SPRING_ERR_TIMEOUT, and the next call on the same context (with
    the default limit) gives the normal result.  No GPU fault is involved: the waits simply stop."""
    from spring_b200 import _lib as L
    from spring_b200.api import SpringError
    N, ctx, info, out, _ = runs
    if N != 8:
        pytest.skip("8^3 mesh only")
    ctx.set_precision("bf16x3")
    ctx.set_option(L.SPRING_OPT_WAIT_POLLS, 0)
    try:
        with pytest.raises(SpringError) as ei:
            ctx.linewidth3(1, ctx.nq0, "gauss", SIGMA)
        assert ei.value.code == L.SPRING_ERR_TIMEOUT
    finally:
        ctx.set_option(L.SPRING_OPT_WAIT_POLLS, -1)
    ctx.synchronize()  # the context and its stream are still usable
    ctx.reset_linewidths()
    lw, _ = ctx.linewidth3(1, ctx.nq0, "gauss", SIGMA)
    ctx.set_precision("fp64")
    np.testing.assert_allclose(lw, out["bf16x3"][0], rtol=1e-12, atol=0.0)


def test_fp64_prescreen_matches_full_fp64(runs):
    """SPRING_OPT_FP64_PRESCREEN: the FP64 kernel on the pre-screened pairs only gives the FP64
    linewidths and phase space of every pair (the dropped pairs' weights are below exp(-40))."""
    from spring_b200 import _lib as L
    N, ctx, info, out, _ = runs
    ctx.set_precision("fp64")
    ctx.set_option(L.SPRING_OPT_FP64_PRESCREEN, 1)
    try:
        ctx.reset_linewidths()
        lw, p3 = ctx.linewidth3(1, ctx.nq0, "gauss", SIGMA)
    finally:
        ctx.set_option(L.SPRING_OPT_FP64_PRESCREEN, 0)
    lw64, p364, _ = out["fp64"]
    np.testing.assert_allclose(lw, lw64, rtol=1e-12, atol=1e-13 * np.abs(lw64).max())
    np.testing.assert_allclose(p3, p364, rtol=1e-10, atol=1e-12 * np.abs(p364).max())
