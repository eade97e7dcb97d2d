"""LineWidth.x path mode on the GPU (through the C ABI) against the CPU oracle."""
import numpy as np
import pytest

from oracle import driver as D
from spring_b200 import synthetic as S
from spring_b200.api import Context, SpringError, from_crystal

pytestmark = pytest.mark.gpu

TEMPS = [100.0, 300.0, 700.0]
# generic segments (no symmetry: no degenerate q0 or q2 modes, so per-mode linewidths do not depend
# on the eigensolver's choice inside a degenerate subspace): one zero-centred, one on the [0, N) mesh
GENERIC = np.array([[0.11, 0.23, 0.37, 0], [0.31, 0.17, 0.05, 3], [0.61, 0.73, 0.57, 0], [0.83, 0.67, 0.91, 2]])
HIGHSYM = np.array([[0.0, 0.0, 0.0, 0], [0.0, 0.5, 0.5, 4], [0.25, 0.625, 0.625, 3], [0.375, 0.75, 0.375, 2],
                    [0.0, 0.0, 0.0, 3], [0.5, 0.5, 0.5, 2]])


@pytest.fixture(scope="module", params=[5, 6])
def setup(request):
    cr = S.build("rocksalt2")
    N = request.param
    st = D.Setup(cr, (N, N, N), TEMPS)
    ctx, _ = from_crystal(cr, (N, N, N), st.temps, phonons={"grid": st.ph, "irr": st.ph0})
    yield st, ctx
    ctx.close()


def test_path_points_match_oracle(setup):
    st, ctx = setup
    q, d, z = ctx.path_qpoints(HIGHSYM)
    qo, do, zo = D.path_points(st.cr.G, HIGHSYM)
    np.testing.assert_allclose(q, qo, rtol=0, atol=1e-14)
    np.testing.assert_allclose(d, do, rtol=1e-15)
    assert np.array_equal(z, zo)


def _generic_points(st):
    q, _, z = D.path_points(st.cr.G, GENERIC[:2])
    q2, _, z2 = D.path_points(st.cr.G, GENERIC[2:])
    return np.concatenate([q, q2]), np.concatenate([z, z2])


@pytest.mark.parametrize("delta", ["tetra", "gauss"])
def test_linewidth_path_matches_oracle(setup, delta):
    st, ctx = setup
    q, z = _generic_points(st)
    assert z.any() and not z.all()
    lw, om = ctx.linewidth_path(q, z, delta=delta, sigma=0.8)
    for k in range(len(q)):
        for it in range(len(TEMPS)):
            ref, info = D.linewidth_path(st, q[k], bool(z[k]), delta, sigma=0.8, it=it)
            assert info["exists"].all()
            scale = np.abs(ref).max()
            np.testing.assert_allclose(lw[it, k], ref, rtol=1e-8, atol=1e-11 * scale)
        np.testing.assert_allclose(om[k], info["omega0"], rtol=1e-12, atol=1e-10)


def test_linewidth_path_high_symmetry_runs(setup):
    """The benchmark path Gamma-X-W-K-Gamma-L: finite, non-negative, degenerate-insensitive sums close."""
    st, ctx = setup
    q, _, z = ctx.path_qpoints(HIGHSYM)
    lw, om = ctx.linewidth_path(q, z, delta="tetra")
    assert np.all(np.isfinite(lw)) and lw.min() >= -1e-12
    k = 3  # X point: the sum over all branches does not depend on the degenerate eigenvector choice
    ref, _ = D.linewidth_path(st, q[k], bool(z[k]), "gauss", sigma=0.8, it=1)
    lg, _ = ctx.linewidth_path(q[k:k + 1], z[k:k + 1], delta="gauss", sigma=0.8)
    np.testing.assert_allclose(lg[1, 0].sum(), ref.sum(), rtol=1e-6)


def test_linewidth_path_errors():
    cr = S.build("rocksalt2")
    ctx = Context(2, (4, 4, 4), 1)
    ctx.set_crystal(cr.latvec, cr.mass)
    with pytest.raises(SpringError) as e:
        ctx.linewidth_path(np.zeros((1, 3)), [1])
    assert e.value.code == 2
    ctx.close()
