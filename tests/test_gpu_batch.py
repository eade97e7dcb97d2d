"""Batched linewidths in one persistent launch (spring_batch_*): several contexts of different
cells, meshes and temperature sets, run together, against each context's own spring_linewidth3
(FP64, same Gaussian formula) and the CPU oracle; the autotuner's choice and graph replays give
the same numbers."""
import numpy as np
import pytest

from oracle import driver as D
from spring_b200 import synthetic as S
from spring_b200.api import Batch, SpringError, from_crystal

pytestmark = pytest.mark.gpu

TEMPS9 = [100.0 * k for k in range(1, 10)]
SIGMA = 0.8


def _workloads():
    out = []
    for name, N, temps in (("rocksalt2", 4, TEMPS9), ("rocksalt2", 5, [300.0, 700.0]), ("rocksalt8", 2, [300.0])):
        cr = S.build(name)
        st = D.Setup(cr, (N, N, N), temps)
        ctx, info = from_crystal(cr, (N, N, N), temps, phonons={"grid": st.ph, "irr": st.ph0})
        out.append((name, N, st, cr, ctx))
    return out


def _close(a, b, rtol):
    scale = max(np.abs(b).max(), 1e-300)
    np.testing.assert_allclose(a, b, rtol=rtol, atol=rtol * 1e-3 * scale)


def test_batch_matches_single_calls_and_oracle():
    wl = _workloads()
    singles = []
    for name, N, temps, cr, ctx in wl:
        ctx.reset_linewidths()
        lw, p3 = ctx.linewidth3(1, ctx.nq0, "gauss", SIGMA)
        singles.append((lw, p3))
    b = Batch()
    idx = []
    for name, N, temps, cr, ctx in wl:
        if name == "rocksalt2" and N == 5:  # two disjoint requests on one context
            h = ctx.nq0 // 2
            idx.append((b.add_linewidth3(ctx, 1, h, SIGMA), 0, h))
            idx.append((b.add_linewidth3(ctx, h + 1, ctx.nq0 - h, SIGMA), h, ctx.nq0))
        else:
            idx.append((b.add_linewidth3(ctx, 1, ctx.nq0, SIGMA), 0, ctx.nq0))
        ctx.reset_linewidths()
    b.run()
    k = 0
    for w, (name, N, temps, cr, ctx) in enumerate(wl):
        lw_ref, p3_ref = singles[w]
        parts = 2 if (name == "rocksalt2" and N == 5) else 1
        for _ in range(parts):
            i, a, e = idx[k]
            lw, p3, ms = b.result(i)
            assert ms > 0.0
            _close(lw, lw_ref[:, a:e], 1e-10)
            _close(p3, p3_ref[a:e], 1e-10)
            k += 1
        # LW_Allq0 was accumulated as spring_linewidth3 does
        _close(ctx.get_linewidths(), lw_ref, 1e-10)
    # one workload against the CPU oracle as well (8-atom cell, Ndof 24, s0 blocks)
    name, N, st, cr, ctx = wl[2]
    lw, _, _ = b.result(idx[-1][0])
    for i0 in range(st.nq0):
        ref = D.linewidth3_q0(st, i0, "gauss", SIGMA, it=0)["lw"]
        np.testing.assert_allclose(lw[0, i0], ref, rtol=1e-8, atol=1e-11 * np.abs(ref).max())
    b.close()
    for *_, ctx in wl:
        ctx.close()


def test_batch_autotuner_and_graph_replay():
    wl = _workloads()
    b = Batch()
    for *_, ctx in wl:
        b.add_linewidth3(ctx, 1, ctx.nq0, SIGMA)
    b.run()
    first = [b.result(i)[0] for i in range(len(wl))]
    cfg, best_ms, tried = b.tune()
    assert tried >= 6 and best_ms > 0.0
    assert cfg[0] in (0, 1) and cfg[1] in (0, 1, 2, 3, 4) and cfg[2] in (6, 12, 24) and cfg[3] in (1, 4, 16)
    assert b.config() == cfg
    for rep in range(2):  # capture with the tuned configuration, then replay
        for *_, ctx in wl:
            ctx.reset_linewidths()
        b.run()
        for i in range(len(wl)):
            _close(b.result(i)[0], first[i], 1e-11)
    # every manual configuration gives the same numbers
    for cfg2 in ((0, 1, 12, 4), (1, 2, 6, 16)):  # every cell in the any-cell layout; two-atom groups
        b.set_config(*cfg2)
        b.run()
        for i in range(len(wl)):
            _close(b.result(i)[0], first[i], 1e-11)
    # a new batch of the same shape starts with the tuned configuration
    b2 = Batch()
    for *_, ctx in wl:
        b2.add_linewidth3(ctx, 1, ctx.nq0, SIGMA)
    b2.run()
    assert b2.config() == cfg
    b2.close()
    b.close()
    for *_, ctx in wl:
        ctx.close()


def test_batch_argument_errors():
    cr = S.build("rocksalt2")
    ctx, _ = from_crystal(cr, (3, 3, 3), [300.0])
    b = Batch()
    with pytest.raises(SpringError):
        b.run()  # empty
    b.add_linewidth3(ctx, 1, 2, SIGMA)
    with pytest.raises(SpringError):
        b.add_linewidth3(ctx, 2, 1, SIGMA)  # overlaps the first request
    with pytest.raises(SpringError):
        b.add_linewidth3(ctx, 1, ctx.nq0 + 1, SIGMA)  # outside the irreducible set
    with pytest.raises(SpringError):
        b.set_config(2, 0, 0, 1)
    b.close()
    # a configuration whose work item does not fit an SM is refused at run time
    cr8 = S.build("rocksalt8")
    ctx8, _ = from_crystal(cr8, (2, 2, 2), [300.0, 600.0])
    b = Batch()
    b.add_linewidth3(ctx8, 1, ctx8.nq0, SIGMA)
    b.set_config(1, 0, 24, 1)
    with pytest.raises(SpringError):
        b.run()
    b.close()
    ctx8.close()
    ctx.close()


def test_batch_tensor_core_requests_and_path_points():
    """A batch mixing a two-atom context set to BF16x3 (run through the tensor-core pass), an FP64
    8-atom context (persistent kernel) and Gaussian path points (launched inside the graph): every
    result equals the context's own single call, on the first run and on a graph replay."""
    cr2, cr8 = S.build("rocksalt2"), S.build("rocksalt8")
    st2 = D.Setup(cr2, (6, 6, 6), [100.0, 300.0, 700.0])
    ctx2, _ = from_crystal(cr2, (6, 6, 6), st2.temps, phonons={"grid": st2.ph, "irr": st2.ph0})
    st8 = D.Setup(cr8, (2, 2, 2), [300.0])
    ctx8, _ = from_crystal(cr8, (2, 2, 2), st8.temps, phonons={"grid": st8.ph, "irr": st8.ph0})
    ctx2.set_precision("bf16x3")
    path = np.array([[0.11, 0.23, 0.37, 0], [0.31, 0.17, 0.05, 5]])
    q, _, z = ctx2.path_qpoints(path)
    singles = []
    for ctx in (ctx2, ctx8):
        ctx.reset_linewidths()
        singles.append(ctx.linewidth3(1, ctx.nq0, "gauss", SIGMA))
    lw_path, om_path = ctx2.linewidth_path(q, z, delta="gauss", sigma=SIGMA)
    b = Batch()
    i2 = b.add_linewidth3(ctx2, 1, ctx2.nq0, SIGMA)
    i8 = b.add_linewidth3(ctx8, 1, ctx8.nq0, SIGMA)
    ip = b.add_path(ctx2, q, z, SIGMA)
    for rep in range(2):
        for ctx in (ctx2, ctx8):
            ctx.reset_linewidths()
        b.run()
        for i, ctx, (lw_ref, p3_ref) in ((i2, ctx2, singles[0]), (i8, ctx8, singles[1])):
            lw, p3, _ = b.result(i)
            _close(lw, lw_ref, 1e-11)
            _close(p3, p3_ref, 1e-11)
            _close(ctx.get_linewidths(), lw_ref, 1e-11)
        lwp, omp = b.path_result(ip)
        _close(lwp, lw_path, 1e-11)
        np.testing.assert_array_equal(omp, om_path)
    b.close()
    ctx2.close()
    ctx8.close()


def test_batch_path_request_errors():
    cr = S.build("rocksalt2")
    ctx, _ = from_crystal(cr, (3, 3, 3), [300.0])
    q = np.zeros((1, 3))
    z = np.ones(1, dtype=np.int32)
    b = Batch()
    with pytest.raises(SpringError):
        b.add_path(ctx, q, z, SIGMA)  # no linewidth request has bound the device yet
    b.add_linewidth3(ctx, 1, 1, SIGMA)
    with pytest.raises(SpringError):
        b.add_path(ctx, q, z, -1.0)
    with pytest.raises(SpringError):
        b.path_result(0)  # no such request
    b.close()
    ctx.close()
