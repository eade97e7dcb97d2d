"""Four-phonon path on the GPU (through the C ABI) against the CPU oracle and the golden quartet lists."""
import numpy as np
import pytest

from oracle import driver as D
from spring_b200 import synthetic as S
from spring_b200.api import Context, SpringError, from_crystal

pytestmark = pytest.mark.gpu

RTOL_RATE = 1e-9   # FP64 rates: summation order and FMA contraction only
TEMPS = [100.0, 300.0, 700.0]


@pytest.fixture(scope="module")
def cr4():
    return S.build("rocksalt2", fc4=True)


@pytest.fixture(scope="module", params=[4, 5])
def setup4(request, cr4):
    N = request.param
    st = D.Setup(cr4, (N, N, N), TEMPS)
    ctx, info = from_crystal(cr4, (N, N, N), st.temps, phonons={"grid": st.ph, "irr": st.ph0}, with_fc4=True)
    yield st, ctx
    ctx.close()


@pytest.mark.parametrize("N", [3, 4])
def test_enumerate4_golden(cr4, golden, N):
    """Identity symmetry, so irreducible point k + 1 is grid point k."""
    ctx = Context(2, (N, N, N), 1)
    ctx.set_crystal(cr4.latvec, cr4.mass)
    ctx.make_mesh(want=False)
    ctx.find_irr_q(np.eye(3, dtype=np.int32)[None])
    for j, k in enumerate(golden[f"enum4_N{N}_q0"]):
        A, Pm, cnt = ctx.enumerate4(int(k) + 1)
        assert cnt == tuple(golden[f"enum4_N{N}_C"][j])
        assert np.array_equal(A, golden[f"enum4_N{N}_A"][j])
        assert np.array_equal(Pm, golden[f"enum4_N{N}_P"][j][: cnt[0]])
    ctx.close()


def test_enumerate4_bit_exact(setup4):
    st, ctx = setup4
    for i0 in range(st.nq0):
        A, Pm, cnt = ctx.enumerate4(i0 + 1)
        Ao, Po, co = D.momentum4(st.mesh, st.q_pnt_int, st.irr_int[i0])
        assert cnt == co
        assert np.array_equal(A, Ao)
        assert np.array_equal(Pm, Po)


def test_enumerate4_cap(setup4):
    st, ctx = setup4
    _, _, cnt = ctx.enumerate4(1)
    with pytest.raises(SpringError) as e:
        ctx.enumerate4(1, cap=cnt[0] - 1)
    assert e.value.code == 1


def _q0_sample(st):
    return sorted({0, 1, st.nq0 - 1})


@pytest.mark.parametrize("delta", ["tetra", "gauss"])
def test_linewidth4_matches_oracle(setup4, delta):
    st, ctx = setup4
    sigma = 0.8
    for i0 in _q0_sample(st):
        rate = ctx.linewidth4(i0 + 1, 1, delta=delta, sigma=sigma)
        for it in range(len(TEMPS)):
            if delta == "tetra":
                ro, _ = D.lw4_tetra(st, i0, it)
            else:
                ro = D.lw4_gauss(st, i0, it, sigma=sigma)
            scale = np.abs(ro).max()
            assert scale > 0
            np.testing.assert_allclose(rate[it, 0], ro, rtol=RTOL_RATE, atol=1e-12 * scale)


def test_linewidth4_block_and_polarization(setup4):
    st, ctx = setup4
    pol = np.array([[2, 6], [4, 6], [1, 6], [3, 5]], np.int32)
    n = min(3, st.nq0)
    rate = ctx.linewidth4(1, n, delta="tetra", pol4=pol)
    for i0 in range(n):
        ro, _ = D.lw4_tetra(st, i0, 1, pol=pol)
        np.testing.assert_allclose(rate[1, i0], ro, rtol=RTOL_RATE, atol=1e-12 * max(np.abs(ro).max(), 1e-30))


def test_linewidth4_adds_half_rate_to_resident(setup4):
    st, ctx = setup4
    ctx.reset_linewidths()
    rate = ctx.linewidth4(2, 1, delta="gauss", sigma=0.8)
    lw = ctx.get_linewidths()
    np.testing.assert_allclose(lw[:, 1], 0.5 * rate[:, 0], rtol=1e-15, atol=0)
    assert not lw[:, [0] + list(range(2, st.nq0))].any()
    ctx.reset_linewidths()


def test_linewidth4_errors(cr4):
    N = 4
    st = D.Setup(cr4, (N, N, N), [300.0])
    ctx, _ = from_crystal(cr4, (N, N, N), st.temps, phonons={"grid": st.ph, "irr": st.ph0}, with_fc4=False)
    with pytest.raises(SpringError) as e:
        ctx.linewidth4(1, 1)
    assert e.value.code == 2
    ctx.set_fc4(cr4.fc4_atm_num, cr4.fc4_atm_indx, cr4.fc4)
    with pytest.raises(SpringError) as e:
        ctx.linewidth4(1, 1, pol4=np.array([[0, 6]] * 4, np.int32))
    assert e.value.code == 1
    with pytest.raises(SpringError) as e:
        ctx.linewidth4(1, 1, delta="gauss", sigma=0.0)
    assert e.value.code == 1
    ctx.close()
