"""Tensor-core (tcgen05) four-phonon V4 with the Gaussian four-phonon rate: BF16 and the compensated
BF16x3 form against the FP64 GPU path (k_v4) and the CPU oracle.  Tolerances are the accuracy targets
of the mixed-precision path: rates of every mode above 1e-3 of the largest within 2e-2 (BF16) and
1e-4 (BF16x3) of FP64; the Gaussian weights, occupations and sums stay FP64 in both."""
import numpy as np
import pytest

from oracle import driver as D
from spring_b200 import synthetic as S
from spring_b200.api import from_crystal

pytestmark = pytest.mark.gpu

TEMPS = [300.0, 700.0]
TOL = {"bf16x3": 1e-4, "bf16": 2e-2}


@pytest.fixture(scope="module")
def cr4():
    return S.build("rocksalt2", fc4=True)


@pytest.fixture(scope="module", params=[4, 5, 6])
def runs(request, cr4):
    N = request.param
    st = D.Setup(cr4, (N, N, N), TEMPS)
    ctx, info = from_crystal(cr4, (N, N, N), st.temps, phonons={"grid": st.ph, "irr": st.ph0}, with_fc4=True)
    out = {}
    for sigma in (0.8, 0.3767):
        for prec in ("fp64", "bf16x3", "bf16"):
            ctx.set_precision(prec)
            out[(prec, sigma)] = ctx.linewidth4(1, ctx.nq0, delta="gauss", sigma=sigma)
    ctx.set_precision("fp64")
    yield N, st, ctx, out
    ctx.close()


def _max_rel(rate, ref):
    e = 0.0
    for it in range(ref.shape[0]):
        big = ref[it] > 1e-3 * ref[it].max()
        e = max(e, float((np.abs(rate[it][big] - ref[it][big]) / ref[it][big]).max()))
    return e


@pytest.mark.parametrize("prec", ["bf16x3", "bf16"])
@pytest.mark.parametrize("sigma", [0.8, 0.3767])
def test_v4tc_rates_vs_fp64(runs, prec, sigma):
    N, st, ctx, out = runs
    ref = out[("fp64", sigma)]
    assert ref.max() > 0
    err = _max_rel(out[(prec, sigma)], ref)
    assert err < TOL[prec], (N, prec, sigma, err)


def test_v4tc_matches_oracle(runs):
    """The compensated tensor-core rates of a few irreducible points against the CPU oracle."""
    N, st, ctx, out = runs
    rate = out[("bf16x3", 0.8)]
    for i0 in sorted({0, 1, st.nq0 - 1}):
        for it in range(len(TEMPS)):
            ro = D.lw4_gauss(st, i0, it, sigma=0.8)
            big = ro > 1e-3 * ro.max()
            assert (np.abs(rate[it, i0][big] - ro[big]) / ro[big]).max() < 1e-4


def test_v4tc_adds_half_rate_to_resident(runs):
    N, st, ctx, out = runs
    ctx.set_precision("bf16x3")
    ctx.reset_linewidths()
    rate = ctx.linewidth4(2, 1, delta="gauss", sigma=0.8)
    lw = ctx.get_linewidths()
    ctx.set_precision("fp64")
    np.testing.assert_allclose(lw[:, 1], 0.5 * rate[:, 0], rtol=1e-15, atol=0)
    assert not lw[:, [0] + list(range(2, st.nq0))].any()
    ctx.reset_linewidths()


def test_v4tc_wait_timeout_returns_status(runs):
    """Every wait of one warp on another in the tensor-core V4 kernel is bounded: with a poll limit
    of 0 each runs out at once, the call fails with SPRING_ERR_TIMEOUT, and the context gives the
    normal result on the next call."""
    from spring_b200 import _lib as L
    from spring_b200.api import SpringError
    N, st, ctx, out = runs
    if N != 4:
        pytest.skip("4^3 mesh only")
    ctx.set_precision("bf16x3")
    ctx.set_option(L.SPRING_OPT_WAIT_POLLS, 0)
    try:
        with pytest.raises(SpringError) as ei:
            ctx.linewidth4(1, 1, delta="gauss", sigma=0.8)
        assert ei.value.code == L.SPRING_ERR_TIMEOUT
    finally:
        ctx.set_option(L.SPRING_OPT_WAIT_POLLS, -1)
    ctx.synchronize()
    rate = ctx.linewidth4(1, ctx.nq0, delta="gauss", sigma=0.8)
    ctx.set_precision("fp64")
    np.testing.assert_allclose(rate, out[("bf16x3", 0.8)], rtol=1e-12, atol=0.0)


def test_v4tc_branch_mask(runs):
    """spring_linewidth4_modes: the selected branches of each q0 equal the full call's, the others
    are zero (the surrogate-screened path spends exact work on selected modes only)."""
    N, st, ctx, out = runs
    ctx.set_precision("bf16x3")
    rng = np.random.default_rng(N)
    mask = rng.integers(0, 64, size=ctx.nq0).astype(np.int32)
    mask[0] = 0x3f
    rate = ctx.linewidth4_modes(1, mask, sigma=0.8)
    ctx.set_precision("fp64")
    full = out[("bf16x3", 0.8)]
    sel = ((mask[:, None] >> np.arange(6)[None, :]) & 1).astype(bool)
    for it in range(len(TEMPS)):
        np.testing.assert_allclose(rate[it][sel], full[it][sel], rtol=1e-12, atol=1e-300)
        assert not rate[it][~sel].any()
