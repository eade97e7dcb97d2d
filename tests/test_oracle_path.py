"""LineWidth.x path-mode oracle (CPU only): path points, the q2 search and a known answer against the
kappa.x-mode oracle at a q0 that lies on the grid."""
import numpy as np
import pytest

from oracle import driver as D
from spring_b200 import synthetic as S

N = 5
PATH = np.array([[0.0, 0.0, 0.0, 0], [0.0, 0.5, 0.5, 4], [0.25, 0.625, 0.625, 3], [0.375, 0.75, 0.375, 2],
                 [0.0, 0.0, 0.0, 3], [0.5, 0.5, 0.5, 2]])


@pytest.fixture(scope="module")
def st():
    return D.Setup(S.build("rocksalt2"), (N, N, N), [300.0])


def test_path_points_reach_every_node(st):
    q, d, z = D.path_points(st.cr.G, PATH)
    counts = PATH[1:, 3].astype(int)
    assert len(q) == counts.sum()
    ends = np.cumsum(counts) - 1
    for k, e in enumerate(ends):
        np.testing.assert_allclose(q[e], st.cr.G @ PATH[k + 1, :3], atol=1e-12)
    assert np.all(np.diff(d) > 0)
    # zero-centred unless neither node is inside [-1/2, 1/2]^3 and none is negative (W -> K here)
    seg = np.repeat(np.arange(len(counts)), counts)
    assert list(z[seg == 2]) == [False] * counts[2] and z[seg != 2].all()


@pytest.mark.parametrize("zero_centered", [True, False])
def test_q2_search_conserves_momentum_inside_the_zone(st, zero_centered):
    q0 = st.cr.G @ np.array([0.13, 0.29, 0.41]) if zero_centered else st.cr.G @ np.array([0.61, 0.73, 0.57])
    _, q1s, _ = D.make_tetrahedron(st.mesh, st.cr.G, zero_centered=zero_centered)
    q2, ex = D.find_q2(st.cr.G, q0, q1s, zero_centered)
    assert ex.all()
    frac = np.linalg.solve(st.cr.G, (q0[None, :] + q1s + q2).T).T
    np.testing.assert_allclose(frac, np.round(frac), atol=1e-10)
    x = np.linalg.solve(st.cr.G, q2.T).T
    if zero_centered:
        assert np.all(np.abs(x) <= 0.5 + 1e-12)
    else:
        assert np.all((x >= -1e-12) & (x <= 1 + 1e-12))


@pytest.mark.parametrize("i0", [1, 4])
def test_gauss_path_at_a_grid_q0_equals_kappa_mode(st, i0):
    """At a q0 on the grid the LineWidth.x Gaussian sum is kappa.x's CalculateLinewidth over every q1
    (same W up to 1/omega vs 1/(omega) products, same deltas): with the same q0 eigenvectors the
    rates agree to rounding."""
    ph0 = {k: (v[:, i0:i0 + 1] if k == "nbe" else v[i0:i0 + 1]) for k, v in st.ph0.items()}
    q0 = st.irr_q[i0]
    lw, info = D.linewidth_path(st, q0, True, "gauss", sigma=0.8, q0_phonons=ph0)
    ref = D.linewidth3_q0(st, i0, "gauss", sigma=0.8)["lw"]
    assert info["exists"].all()
    np.testing.assert_allclose(lw, ref, rtol=1e-9, atol=1e-12 * np.abs(ref).max())


def test_tetra_path_generic_point_is_finite_and_positive(st):
    q0 = st.cr.G @ np.array([0.13, 0.29, 0.41])
    lw, info = D.linewidth_path(st, q0, True, "tetra")
    assert np.all(np.isfinite(lw)) and lw.min() > 0
