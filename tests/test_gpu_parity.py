"""GPU library (through the C ABI) against the CPU oracle and the golden fixtures."""
import numpy as np
import pytest

from oracle import driver as D
from spring_b200 import synthetic as S
from spring_b200.api import Context, SpringError, from_crystal

pytestmark = pytest.mark.gpu

RTOL_LW = 1e-9      # FP64 linewidths: summation order and FMA contraction only


@pytest.fixture(scope="module")
def cr():
    return S.build("rocksalt2")


def _oracle_phonons(st):
    return {"grid": st.ph, "irr": st.ph0}


@pytest.fixture(scope="module", params=[5, 8])
def pair(request, cr):
    N = request.param
    st = D.Setup(cr, (N, N, N), [100.0, 300.0, 700.0])
    ctx, info = from_crystal(cr, (N, N, N), st.temps, phonons=_oracle_phonons(st))
    yield st, ctx, info
    ctx.close()


def test_mesh_and_irreducible_set(pair):
    st, ctx, info = pair
    assert np.array_equal(info["q_pnt_int"], st.q_pnt_int)
    assert np.array_equal(info["tetra"], st.tetra)
    np.testing.assert_allclose(info["q_pnt"], st.q_pnt, rtol=0, atol=1e-14)
    assert np.array_equal(info["irr_q_pnt_int"], st.irr_int)
    assert np.array_equal(info["pos"], st.pos)
    assert np.array_equal(info["multiplicity"], st.mult)


def test_enumerate3_bit_exact(pair):
    st, ctx, _ = pair
    for i0 in range(st.nq0):
        A, Pm, cnt = ctx.enumerate3(i0 + 1)
        Ao, Po, co = D.momentum3(st.mesh, st.q_pnt_int, st.irr_int[i0])
        assert cnt == co
        assert np.array_equal(A, Ao)
        assert np.array_equal(Pm, Po)


@pytest.mark.parametrize("N", [4, 6])
def test_enumerate3_golden_every_q0(cr, golden, N):
    """Every grid point as q0 (identity symmetry only), against the Python transcription."""
    ctx = Context(2, (N, N, N), 1)
    ctx.set_crystal(cr.latvec, cr.mass)
    ctx.make_mesh(want=False)
    ctx.find_irr_q(np.eye(3, dtype=np.int32)[None])
    assert ctx.nq0 == N ** 3
    for k in range(N ** 3):
        A, Pm, cnt = ctx.enumerate3(k + 1)
        assert cnt == tuple(golden[f"enum3_N{N}_C"][k])
        assert np.array_equal(A, golden[f"enum3_N{N}_A"][k])
        assert np.array_equal(Pm, golden[f"enum3_N{N}_P"][k][: cnt[0]])
    ctx.close()


@pytest.mark.parametrize("generic", [False, True])
def test_scatter_w3(pair, generic):
    st, ctx, _ = pair
    ctx.use_generic_v3(generic)
    for i0 in (0, 1, st.nq0 - 1):
        r = D.linewidth3_q0(st, i0, with_w=True)
        w = ctx.scatter_w3(i0 + 1)
        scale = r["sctr"].max()
        np.testing.assert_allclose(w, r["sctr"], rtol=1e-9, atol=1e-12 * scale)
    ctx.use_generic_v3(False)


@pytest.mark.parametrize("delta", ["gauss", "tetra"])
@pytest.mark.parametrize("generic", [False, True])
def test_linewidth3_all_q0(pair, delta, generic):
    st, ctx, _ = pair
    ctx.use_generic_v3(generic)
    ctx.reset_linewidths()
    lw, p3 = ctx.linewidth3(1, st.nq0, delta=delta, sigma=0.3767)
    ref = D.linewidth3_all(st, delta, 0.3767)
    np.testing.assert_allclose(lw, ref, rtol=RTOL_LW, atol=1e-14 * np.abs(ref).max())
    # the resident LW_Allq0 holds the same
    np.testing.assert_allclose(ctx.get_linewidths(), lw, rtol=0, atol=0)
    for i0 in (0, st.nq0 // 2):
        r = D.linewidth3_q0(st, i0, delta=delta, sigma=0.3767)
        np.testing.assert_allclose(p3[i0], r["p3_q0"], rtol=1e-10, atol=1e-14 * max(1.0, np.abs(r["p3_q0"]).max()))
    ctx.use_generic_v3(False)


def test_linewidth3_polarization_window(pair):
    st, ctx, _ = pair
    pol = np.array([[4, 6], [1, 3], [1, 6]], np.int32)   # Polarization3rd(2,3) memory: (lo,hi) per column
    lw, _ = ctx.linewidth3(1, st.nq0, delta="tetra", pol3=pol)
    i0 = min(2, st.nq0 - 1)
    r = D.linewidth3_q0(st, i0, delta="tetra", pol=pol, it=1)
    np.testing.assert_allclose(lw[1, i0], r["lw"], rtol=RTOL_LW, atol=1e-14 * np.abs(r["lw"]).max())


@pytest.mark.parametrize("delta", ["gauss", "tetra"])
def test_isotope_rate(pair, delta):
    st, ctx, _ = pair
    g2 = np.array([1e-3, 1e-3])
    rate = ctx.linewidth_iso(1, st.nq0, g2, delta=delta, sigma=0.3767)
    for i0 in (0, st.nq0 - 1):
        wi = D.iso_w(2, st.ph0["evec"][i0], st.ph0["omega"][i0], st.ph["evec"], g2)
        ref = (D.iso_lw_gauss(st.ph0["omega"][i0], st.ph["omega"], wi, 0.3767) if delta == "gauss"
               else D.iso_lw_tetra(st.ph0["omega"][i0], st.ph["omega"], wi, st.tetra))
        for t in range(3):
            np.testing.assert_allclose(rate[t, i0], ref, rtol=1e-9, atol=1e-14 * max(1e-30, np.abs(ref).max()))


@pytest.mark.parametrize("symm", [True, False])
def test_kappa_rta(pair, symm):
    st, ctx, info = pair
    ctx.reset_linewidths()
    ctx.linewidth3(1, st.nq0, delta="tetra", want=False)
    kap = ctx.kappa_rta(info["Rxyz"], symm=symm)
    lw = ctx.get_linewidths()
    ref = D.kappa_rta(st, lw, symm=symm)
    np.testing.assert_allclose(kap, ref, rtol=1e-11, atol=1e-13 * np.abs(ref).max())


def test_device_phonons_gauge_invariants(cr):
    """The device eigensolver against LAPACK zheevd: frequencies, velocities of non-degenerate
    modes, eigen-projectors and occupations."""
    N = 6
    st = D.Setup(cr, (N, N, N), [300.0])
    ctx, _ = from_crystal(cr, (N, N, N), st.temps, phonons="device")
    for which, ref in ((0, st.ph), (1, st.ph0)):
        ph = ctx.get_phonons(which)
        # compare eigenvalues (omega^2): omega = sqrt|lambda| amplifies the round-off of the
        # zero eigenvalues at Gamma (1e-15 of the spectrum -> 1e-6 rad/ps)
        np.testing.assert_allclose(np.sign(ph["omega"]) * ph["omega"] ** 2,
                                   np.sign(ref["omega"]) * ref["omega"] ** 2, rtol=1e-10, atol=1e-10)
        np.testing.assert_allclose(ph["nbe"], ref["nbe"], rtol=1e-8, atol=1e-12)
        for q in range(ref["omega"].shape[0]):
            w = ref["omega"][q]
            for s in range(6):
                gap = np.min(np.abs(np.delete(w, s) - w[s]))
                if gap < 1e-3 * max(1.0, abs(w[s])) or abs(w[s]) < 1e-3:
                    continue
                e, f = ph["evec"][q, s], ref["evec"][q, s]
                np.testing.assert_allclose(np.outer(e, e.conj()), np.outer(f, f.conj()), atol=1e-9)
                np.testing.assert_allclose(ph["grp_vel"][q, s], ref["grp_vel"][q, s], rtol=1e-7, atol=1e-6)
    ctx.close()


def test_end_to_end_device_phonons_kappa(cr):
    """Whole path with device phonons: kappa within 1e-6 of the oracle (LAPACK phonons)."""
    N = 8
    st = D.Setup(cr, (N, N, N), [300.0])
    ctx, info = from_crystal(cr, (N, N, N), st.temps, phonons="device")
    ctx.linewidth3(1, st.nq0, delta="tetra", want=False)
    kap = ctx.kappa_rta(info["Rxyz"])[0]
    ref = D.kappa_rta(st, D.linewidth3_all(st, "tetra"))[0]
    np.testing.assert_allclose(kap[[0, 4, 8]], ref[[0, 4, 8]], rtol=1e-6)
    ctx.close()


def test_errors_are_reported(cr):
    ctx = Context(2, (4, 4, 4), 1)
    with pytest.raises(SpringError) as e:
        ctx.linewidth3(1, 1)
    assert e.value.code == 2  # SPRING_ERR_STATE
    ctx.set_crystal(cr.latvec, cr.mass)
    ctx.make_mesh(want=False)
    ctx.find_irr_q(S.point_group(cr)[0])
    with pytest.raises(SpringError) as e:
        ctx.linewidth3(0, 1)
    assert e.value.code == 1  # SPRING_ERR_ARG
    with pytest.raises(SpringError) as e:
        ctx.linewidth3(1, ctx.nq0 + 1)
    assert e.value.code == 1
    ctx.close()


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_fault_injection_clean_error(cr, kind):
    """An injected allocation / copy / launch failure surfaces as an error and the context stays usable."""
    N = 4
    st = D.Setup(cr, (N, N, N), [300.0])
    ctx, info = from_crystal(cr, (N, N, N), st.temps, phonons=_oracle_phonons(st))
    ctx.inject_fault(kind, 1)
    with pytest.raises(SpringError) as e:
        ctx.linewidth3(1, st.nq0, delta="tetra")
    assert e.value.code == 6
    lw, _ = ctx.linewidth3(1, st.nq0, delta="tetra")
    ref = D.linewidth3_all(st, "tetra")
    np.testing.assert_allclose(lw, ref, rtol=RTOL_LW, atol=1e-14 * np.abs(ref).max())
    ctx.close()
