"""Four-phonon oracle: V4 in the reference loop order vs the regrouped form, and the rate identities
the device kernels rely on (CPU only)."""
import numpy as np
import pytest

from oracle import driver as D
from spring_b200 import synthetic as S

N = 4
PER = np.array([[0, 2, 1], [1, 0, 2], [1, 2, 0], [2, 0, 1], [2, 1, 0]])  # Permutation4th, 0-based


@pytest.fixture(scope="module")
def st4():
    cr = S.build("rocksalt2", fc4=True)
    return D.Setup(cr, (N, N, N), [300.0])


def _naive(st, i0, g):
    q0chk = np.array([all(st.irr_int[i0] == 0)] + [all(st.q_pnt_int[x] == 0) for x in g], np.int32)
    return D.w4_naive(st.cr, st.nq, st.q_pnt[g[0]], st.q_pnt[g[1]], st.q_pnt[g[2]], q0chk,
                      st.ph0["evec"][i0], st.ph0["onebyomega"][i0],
                      st.ph["evec"][g[0]], st.ph["onebyomega"][g[0]], st.ph["evec"][g[1]], st.ph["onebyomega"][g[1]],
                      st.ph["evec"][g[2]], st.ph["onebyomega"][g[2]])


@pytest.mark.parametrize("i0", [0, 1, 3])
def test_w4_regrouped_matches_reference_loop_order(st4, i0):
    """ScatterMatEl4 + ScatterProbability4 (FourthOrder_m.f90:286-473) vs the basis-block regrouping."""
    _, perm, _ = D.momentum4(st4.mesh, st4.q_pnt_int, st4.irr_int[i0])
    pick = perm[[0, 1, len(perm) // 2, len(perm) - 1]]
    Wf = D.w4_factored(st4, i0, pick)
    for k, q in enumerate(pick):
        Wn = _naive(st4, i0, q - 1)
        scale = np.abs(Wn).max()
        assert scale > 0
        np.testing.assert_allclose(Wf[k], Wn, rtol=1e-11, atol=1e-13 * scale)


def test_w4_symmetric_under_reordering(st4):
    """FC4 symmetric in its three neighbour slots => W(q0; qa sa, qb sb, qc sc) is symmetric in the
    (q, s) pairs.  The Gaussian device kernel reads every ordering from its quartet's W on this basis."""
    i0 = 1
    _, perm, _ = D.momentum4(st4.mesh, st4.q_pnt_int, st4.irr_int[i0])
    q = perm[[3, 40, 200]]
    W = D.w4_factored(st4, i0, q)
    for p in PER:
        Wp = D.w4_factored(st4, i0, q[:, p])
        np.testing.assert_allclose(Wp, W.transpose(0, 1, *(2 + p)), rtol=1e-11, atol=1e-13 * np.abs(W).max())


def test_lw4_gauss_equals_quartet_form(st4):
    """The oracle's Gaussian rate (W computed directly for every ordered (q1, q2)) equals the same sum
    taken over quartets with each ordering's W read from the quartet through the exact inverse of its
    permutation - the summation the fused device kernel performs."""
    i0, sigma = 1, 0.8
    A, perm, _ = D.momentum4(st4.mesh, st4.q_pnt_int, st4.irr_int[i0])
    Wq = D.w4_factored(st4, i0, perm)
    ref = D.lw4_gauss(st4, i0, 0, sigma=sigma)
    om0, n0 = st4.ph0["omega"][i0], st4.ph0["nbe"][0][i0]
    om, nb = st4.ph["omega"], st4.ph["nbe"][0]
    rate = np.zeros(st4.cr.ndof)
    pre = 1.0 / sigma / np.sqrt(2.0 * np.pi)
    for q1 in range(st4.nq):
        for q2 in range(st4.nq):
            typ, pos, q3 = A[q1, q2]
            W = Wq[pos - 1]
            if typ > 0:
                W = W.transpose(0, *(1 + PER[typ - 1]))
            q3 -= 1
            w1, w2, w3 = om[q1][:, None, None], om[q2][None, :, None], om[q3][None, None, :]
            n1, n2, n3 = nb[q1][:, None, None], nb[q2][None, :, None], nb[q3][None, None, :]
            for s0 in range(3 if all(st4.irr_int[i0] == 0) else 0, st4.cr.ndof):
                d1, d2, d3 = om0[s0] - (w1 + w2 + w3), om0[s0] - (w2 + w3 - w1), om0[s0] - (w3 - w1 - w2)
                g = lambda d: pre * np.exp(-0.5 * (d / sigma) ** 2)
                rate[s0] += np.sum(W[s0] * (n1 * n2 * n3 / n0[s0] * g(d1) / 6.0
                                            + (1 + n1) * n2 * n3 / n0[s0] * g(d2) / 2.0
                                            + (1 + n1) * (1 + n2) * n3 / n0[s0] * g(d3) / 2.0))
    np.testing.assert_allclose(rate, ref, rtol=1e-10, atol=1e-14 * np.abs(ref).max())


def test_lw4_tetra_reads_quartets_through_reference_permutation(st4):
    """TetrahedronIntegration4th takes after_perm = before_perm(per(:, type)): for the two 3-cycles
    (types 3 and 4) that is the inverse of the exact mapping.  The oracle keeps the reference's
    reading; with W symmetric the rates are finite, non-negative and not all zero."""
    i0 = 1
    rate, info = D.lw4_tetra(st4, i0, 0)
    assert np.all(np.isfinite(rate)) and np.all(rate >= 0) and rate.max() > 0
    typ = info["Allq1q2q3"][..., 0]
    assert {3, 4} & set(np.unique(typ).tolist())  # the 3-cycle types occur on this mesh
