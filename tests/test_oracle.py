"""The C++ FP64 oracle against the golden fixtures and the reference's own invariants (CPU only)."""
import numpy as np
import pytest

from oracle import driver as D
from oracle import constants as C
from spring_b200 import synthetic as S


@pytest.fixture(scope="module")
def cr():
    return S.build("rocksalt2")


def test_make_tetrahedron_matches_golden(cr, golden):
    for N in (4, 5):
        qi, qf, tet = D.make_tetrahedron((N, N, N), cr.G)
        assert np.array_equal(qi, golden[f"mesh{N}_qint"])
        assert np.array_equal(tet, golden[f"mesh{N}_tet"])
        np.testing.assert_allclose(qf, golden[f"mesh{N}_qpnt"], rtol=0, atol=1e-14)


def test_mesh_invariants(cr):
    N = 6
    qi, qf, tet = D.make_tetrahedron((N, N, N), cr.G)
    assert tet.shape == (6 * N ** 3, 4)
    assert set(np.unique(tet)) == set(range(1, N ** 3 + 1))
    assert qi.min() == -N // 2 + 1 and qi.max() == N // 2
    # every grid point is a vertex of 24 tetrahedra
    assert np.all(np.bincount(tet.ravel())[1:] == 24)


@pytest.mark.parametrize("N,expected", [(8, 29), (12, 72), (16, 145)])
def test_irreducible_counts_fcc(cr, N, expected):
    """Known answers: Gamma-centred N^3 fcc mesh under the 48 operations of O_h."""
    qi, _, _ = D.make_tetrahedron((N, N, N), cr.G)
    W, _ = S.point_group(cr)
    assert len(W) == 48
    ir = D.irr_q((N, N, N), W, qi)
    assert ir["irr_q_pnt_int"].shape[0] == expected
    assert ir["multiplicity"].sum() == N ** 3
    # representatives are the smallest grid index of their orbit, in ascending order
    reps = np.flatnonzero(ir["map"] == np.arange(N ** 3))
    assert np.array_equal(qi[reps], ir["irr_q_pnt_int"])


@pytest.mark.parametrize("N", [4, 5, 6])
def test_enumerate3_matches_golden(cr, golden, N):
    qi, _, _ = D.make_tetrahedron((N, N, N), cr.G)
    A_g, P_g, C_g = golden[f"enum3_N{N}_A"], golden[f"enum3_N{N}_P"], golden[f"enum3_N{N}_C"]
    for k, q0 in enumerate(qi):
        A, Pm, cnt = D.momentum3((N, N, N), qi, q0)
        assert cnt == tuple(C_g[k])
        assert np.array_equal(A, A_g[k])
        assert np.array_equal(Pm, P_g[k][: cnt[0]])


@pytest.mark.parametrize("N", [5, 7, 11])
def test_enumerate3_odd_mesh_closed_form(cr, N):
    """The reference's own assertion (QuasiMomentumConsrv3rd_m.f90:148): Nq/2+1 pairs, Nq covered."""
    qi, _, _ = D.make_tetrahedron((N, N, N), cr.G)
    nq = N ** 3
    for q0 in qi[:: max(1, nq // 40)]:
        _, _, cnt = D.momentum3((N, N, N), qi, q0)
        assert cnt == (nq // 2 + 1, nq)


@pytest.mark.parametrize("N", [3, 4])
def test_enumerate4_matches_golden(cr, golden, N):
    qi, _, _ = D.make_tetrahedron((N, N, N), cr.G)
    for j, k in enumerate(golden[f"enum4_N{N}_q0"]):
        A, Pm, cnt = D.momentum4((N, N, N), qi, qi[k])
        assert cnt == tuple(golden[f"enum4_N{N}_C"][j])
        assert np.array_equal(A, golden[f"enum4_N{N}_A"][j])
        assert np.array_equal(Pm, golden[f"enum4_N{N}_P"][j][: cnt[0]])


def test_enumerate4_odd_mesh_closed_form(cr):
    """QuasiMomentumConsrv4th_m.f90:190: Nq^2/6 + Nq/2 + 1 quartets and Nq^2 covered on a prime mesh."""
    N = 5
    qi, _, _ = D.make_tetrahedron((N, N, N), cr.G)
    nq = N ** 3
    for q0 in qi[[0, 7, 60]]:
        _, _, cnt = D.momentum4((N, N, N), qi, q0)
        assert cnt == ((nq * nq) // 6 + nq // 2 + 1, nq * nq)


@pytest.mark.parametrize("strict", [0, 1])
def test_find_g_iver_matches_golden(golden, strict):
    for k in range(len(golden["giver_Mqs"])):
        e, g, I, Ms, Fs, perm = D.find_g_iver(golden["giver_Mqs"][k], golden["giver_M"][k], golden["giver_F"][k],
                                              strict)
        assert e == bool(golden[f"giver{strict}_e"][k])
        np.testing.assert_array_equal(Ms, golden[f"giver{strict}_Ms"][k])
        np.testing.assert_array_equal(perm, golden[f"giver{strict}_perm"][k])
        np.testing.assert_array_equal(Fs, golden[f"giver{strict}_Fs"][k])
        np.testing.assert_allclose(g, golden[f"giver{strict}_g"][k], rtol=1e-13, equal_nan=True)
        np.testing.assert_allclose(I, golden[f"giver{strict}_I"][k], rtol=1e-12, atol=1e-13, equal_nan=True)


def test_tetrahedron_weights_known_answers():
    """Sum of I_v is 1 (TetrahedronIntegration_m.f90:207) and a linear F is integrated exactly."""
    rng = np.random.default_rng(5)
    for _ in range(300):
        M = rng.normal(0, 1, 4)
        Mqs = rng.uniform(M.min(), M.max())
        a, b = rng.normal(size=2)
        e, g, I, Ms, Fs, perm = D.find_g_iver(Mqs, M, a + b * M)
        assert e and g > 0
        assert abs(I.sum() - 1.0) < 1e-12
        assert abs(np.dot(I, Fs) - (a + b * Mqs)) < 1e-10 * (1 + abs(a) + abs(b))
    # the tetrahedron DOS integrates to one
    M = np.array([0.1, 0.45, 0.8, 1.7])
    xs = np.linspace(0.1, 1.7, 20001)
    gs = [D.find_g_iver(x, M, np.ones(4))[1] for x in xs]
    assert abs(np.trapezoid(gs, xs) - 1.0) < 1e-6


def test_scatter_w3_matches_golden(golden):
    """The oracle's W3 against the 9-deep Python transcription of ScatterMatEl, same inputs."""
    N = 4
    cr = S.Crystal("g", golden["v3_latvec"], np.zeros((2, 3)), np.array([1, 2]), golden["v3_mass"])
    cr.fc3, cr.fc3_atm_num, cr.fc3_atm_indx = golden["v3_fc3"], golden["v3_fc3_num"], golden["v3_fc3_idx"]
    qi, qf, _ = D.make_tetrahedron((N, N, N), cr.G)
    ev, ob = golden["v3_evec"], golden["v3_onebyomega"]
    pairs = golden["v3_pairs"]
    sctr = D.scatter_w3(cr, qf, qi, golden["v3_q0int"], ev[0], ob[0], ev[1:], ob[1:], pairs)
    for k, (g1, g2) in enumerate(pairs):
        ref = golden["v3_W"][k]
        scale = ref.max()
        np.testing.assert_allclose(sctr[g1 - 1], ref, rtol=1e-9, atol=1e-12 * scale)
        if g1 != g2:
            np.testing.assert_allclose(sctr[g2 - 1], ref.transpose(0, 2, 1), rtol=1e-9, atol=1e-12 * scale)


@pytest.fixture(scope="module")
def setup5(cr):
    return D.Setup(cr, (5, 5, 5), [300.0])


def test_w3_invariants(setup5):
    """W is gauge invariant, q1<->q2 symmetric, and zero for Gamma acoustic modes."""
    st = setup5
    i0 = 1
    r = D.linewidth3_q0(st, i0, with_w=True)
    sctr, A = r["sctr"], r["Allq1q2"]
    for g1 in range(st.nq):
        g2 = A[g1, 3] - 1
        np.testing.assert_allclose(sctr[g2], sctr[g1].transpose(0, 2, 1), rtol=1e-10, atol=1e-14 * sctr.max())
    # q1 = Gamma (grid index 1): its acoustic modes s1 <= 3 carry no weight
    assert np.all(sctr[0][:, :3, :] == 0.0) and np.abs(sctr[0][:, 3:, :]).max() > 0.0
    # random phases on every eigenvector leave W unchanged
    rng = np.random.default_rng(1)
    ev = st.ph["evec"] * np.exp(1j * rng.uniform(0, 2 * np.pi, st.ph["evec"].shape[:2]))[:, :, None]
    ev0 = st.ph0["evec"][i0] * np.exp(1j * rng.uniform(0, 2 * np.pi, st.cr.ndof))[:, None]
    s2 = D.scatter_w3(st.cr, st.q_pnt, st.q_pnt_int, st.irr_int[i0], ev0, st.ph0["onebyomega"][i0], ev,
                      st.ph["onebyomega"], r["perm"])
    np.testing.assert_allclose(s2, sctr, rtol=1e-9, atol=1e-13 * sctr.max())


def test_asr_gamma_acoustic_vanishes(setup5):
    """With FC3 obeying the acoustic sum rule, Phi vanishes when q2 is a Gamma acoustic mode."""
    st = setup5
    cr = st.cr
    # e2 = rigid translation (sqrt(m) u) at Gamma, contracted by hand with the factored form
    u = np.array([0.3, -0.5, 0.8])
    rsm = 1.0 / np.sqrt(cr.mass)
    for mu in range(cr.nbasis):
        # sum_{N2,c} FC3(mu,N1,N2,a,b,c) * m_eta^-1/2 * sqrt(m_eta) u_c = sum_N2 FC3 . u
        t = np.einsum("nkabc,c->nab", cr.fc3[mu], u)
        assert np.abs(t).max() < 1e-10
    assert rsm.shape == (2,)


def test_gaussian_matches_direct_sum(setup5):
    """orc_lw3_gauss equals a numpy restatement of CalculateLinewidth over every q1."""
    st = setup5
    i0 = 3
    r = D.linewidth3_q0(st, i0, delta="gauss", sigma=0.8, with_w=True)
    sctr, A = r["sctr"], r["Allq1q2"]
    om0 = st.ph0["omega"][i0]
    om, nb = st.ph["omega"], st.ph["nbe"][0]
    lw = np.zeros(6)
    for q1 in range(st.nq):
        q2 = A[q1, 3] - 1
        o1, o2 = om[q1][:, None], om[q2][None, :]
        n1, n2 = nb[q1][:, None], nb[q2][None, :]
        for s0 in range(6):
            d = lambda x: np.exp(-0.5 * (x / 0.8) ** 2) / (0.8 * np.sqrt(2 * np.pi))
            lw[s0] += np.sum(sctr[q1][s0] * ((n1 + n2 + 1) * d(om0[s0] - o1 - o2) +
                                             (n1 - n2) * (d(om0[s0] + o1 - o2) - d(om0[s0] - o1 + o2))))
    np.testing.assert_allclose(r["lw"], lw, rtol=1e-11)


def test_kappa_cubic_isotropy(setup5):
    st = setup5
    lw = D.linewidth3_all(st, "tetra")
    kap = D.kappa_rta(st, lw, symm=True)[0]
    assert kap[0] > 0
    np.testing.assert_allclose(kap[[4, 8]], kap[0], rtol=1e-12)
    assert np.abs(kap[[1, 2, 3, 5, 6, 7]]).max() < 1e-10 * kap[0]
    full = D.kappa_rta(st, lw, symm=False)[0]
    # the full-grid sum and the symmetrised sum agree up to the FC2 noise anisotropy
    assert abs(np.trace(full.reshape(3, 3)) / 3 - kap[0]) < 0.05 * kap[0]


def test_bte_iteration0_is_full_grid_rta(cr):
    """kappa_iter's 1/tau equals twice kappa.x's linewidth per mode, and its iteration-0 kappa
    equals kappa.x's full-grid RTA kappa, when both use every grid point (identity symmetry)."""
    N = 4
    st = D.Setup(cr, (N, N, N), [300.0], W=np.eye(3, dtype=np.int32)[None], Rxyz=np.eye(3)[None])
    r = D.bte_iter(st)
    lw = D.linewidth3_all(st, "tetra")
    np.testing.assert_allclose(r["inv_tau"], 2.0 * lw[0][r["irr_grid"]], rtol=1e-10, atol=1e-16)
    kf = D.kappa_rta(st, lw, symm=False)[0]
    np.testing.assert_allclose(r["kappa_rta"], kf, rtol=1e-10, atol=1e-10 * np.abs(kf).max())
    assert r["iters"] > 1 and r["kappa"][0] > r["kappa_rta"][0]


def test_bte_gauss_iteration0_is_gaussian_linewidth(cr):
    """The Gaussian operator's 1/tau is twice kappa.x's Gaussian linewidth per mode (full grid), and
    the iteration converges above the RTA start."""
    N, sigma = 4, 1.5
    st = D.Setup(cr, (N, N, N), [300.0], W=np.eye(3, dtype=np.int32)[None], Rxyz=np.eye(3)[None])
    r = D.bte_iter_gauss(st, sigma)
    lw = D.linewidth3_all(st, "gauss", sigma=sigma)
    np.testing.assert_allclose(r["inv_tau"], 2.0 * lw[0][r["irr_grid"]], rtol=1e-10, atol=1e-16)
    assert 1 < r["iters"] < 1000 and r["kappa"][0] > r["kappa_rta"][0]


def test_constants():
    assert abs(C.wTHz - 98.22693) < 1e-4
    assert abs(0.3767 - 2 * 2 * np.pi * 2.99792458e-2) < 2e-4   # 2 cm^-1 in rad/ps
