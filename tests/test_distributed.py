"""The multi-rank path on CPU ranks (gloo, world size 2): the q0 partition, each rank's block of
linewidths, the all-reduce of the zero-padded LW_Allq0 (the reference's co_sum,
src/Kappa/Src/main.f90:677-683) and the all-gather of a per-iteration field, against one process.
The linewidths come from the CPU oracle here (no GPU on these ranks); on GPUs the same calls move the
library's device results over NCCL."""
import os
import socket
import tempfile

import numpy as np
import pytest

from spring_b200 import distributed as DD

N = 5
TEMPS = [300.0, 700.0]


def test_distribute_qpoints_is_the_reference_split():
    # DistributeQpoints: the first mod(Nqs, Nprocs) images take one more, edges 1-based
    for nqs, world in ((29, 2), (29, 4), (413, 8), (3, 4)):
        sizes, edges = [], []
        for rank in range(world):
            size, off, (e1, e2) = DD.distribute_qpoints(nqs, world, rank)
            assert off == e1 - 1 and e2 - e1 + 1 == size
            sizes.append(size)
            edges.append((e1, e2))
        assert sum(sizes) == nqs and max(sizes) - min(sizes) <= 1
        assert sizes == sorted(sizes, reverse=True)
        assert edges[0][0] == 1 and all(edges[k + 1][0] == edges[k][1] + 1 for k in range(world - 1))


def test_partition_by_cost_tiles_and_balances():
    rng = np.random.default_rng(3)
    costs = rng.integers(50, 300, size=413)
    for world in (1, 2, 3, 8):
        blocks = [DD.partition_by_cost(costs, world, r) for r in range(world)]
        assert blocks[0][0] == 0 and blocks[-1][1] == len(costs)
        assert all(blocks[k][1] == blocks[k + 1][0] for k in range(world - 1))
        share = [costs[lo:hi].sum() for lo, hi in blocks]
        assert max(share) - min(share) <= 2 * costs.max()


def _rank_main(rank, world, port, outdir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from oracle import driver as D
        from spring_b200 import synthetic as S
        cr = S.build("rocksalt2")
        st = D.Setup(cr, (N, N, N), TEMPS)
        counts = [D.momentum3(st.mesh, st.q_pnt_int, st.irr_int[i])[2][0] for i in range(st.nq0)]
        lo, hi = DD.partition_by_cost(counts, world, rank)
        mine = D.linewidth3_all(st, "gauss", 0.8, q0_list=range(lo, hi))[:, lo:hi]
        full = DD.allreduce_linewidths(mine, lo, hi, st.nq0)
        kap = D.kappa_rta(st, full)
        # a per-iteration field F(q0, s, 3), gathered along q0 from the ranks' blocks
        F = np.arange(st.nq0 * cr.ndof * 3, dtype=np.float64).reshape(st.nq0, cr.ndof, 3) * 0.5 + rank * 0
        Fg = DD.allgather_blocks(F[lo:hi], lo, hi, st.nq0, axis=0)
        np.savez(os.path.join(outdir, f"r{rank}.npz"), lw=full, kappa=kap, F=Fg, block=np.array([lo, hi]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_ranks_match_one_process():
    import torch.multiprocessing as mp
    from oracle import driver as D
    from spring_b200 import synthetic as S
    world = 2
    with tempfile.TemporaryDirectory() as outdir:
        mp.start_processes(_rank_main, args=(world, _free_port(), outdir), nprocs=world, join=True,
                           start_method="spawn")
        res = [np.load(os.path.join(outdir, f"r{r}.npz")) for r in range(world)]
    cr = S.build("rocksalt2")
    st = D.Setup(cr, (N, N, N), TEMPS)
    lw1 = D.linewidth3_all(st, "gauss", 0.8)
    k1 = D.kappa_rta(st, lw1)
    blocks = [tuple(r["block"]) for r in res]
    assert blocks[0][0] == 0 and blocks[0][1] == blocks[1][0] and blocks[1][1] == st.nq0
    assert 0 < blocks[0][1] < st.nq0  # both ranks own work
    for r in res:
        np.testing.assert_allclose(r["lw"], lw1, rtol=1e-13, atol=0)
        np.testing.assert_allclose(r["kappa"], k1, rtol=1e-12, atol=1e-14 * np.abs(k1).max())
        F = np.arange(st.nq0 * cr.ndof * 3, dtype=np.float64).reshape(st.nq0, cr.ndof, 3) * 0.5
        np.testing.assert_array_equal(r["F"], F)
