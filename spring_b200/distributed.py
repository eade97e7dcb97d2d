"""Multi-rank plumbing of the scattering path: one process per GPU, torch.distributed for the exchange.

The reference distributes the irreducible q0 over coarray images (DistributeQpoints,
src/Kappa/Src/Helper_m.f90:356-434), lets each image compute the linewidths of its block, and sums
the zero-padded LW_Allq0 with co_sum before kappa (src/Kappa/Src/main.f90:677-683).  The iterative
solver (src/Kappa/Src_iterative/main.f90:257-325) exchanges the distribution F(3, Ndof, Nq0) of
every image once per iteration in the same way.  Here the blocks are contiguous ranges of
irreducible points, either the reference's equal-count split or a split balanced by cost (pairs
or quartets per q0), and the exchanges are collectives of the process group (NCCL between GPUs,
gloo on CPU): an all-reduce of the zero-padded block, or an all-gather of the blocks.
"""
from __future__ import annotations

import numpy as np


def distribute_qpoints(nqs: int, world: int, rank: int):
    """The reference's DistributeQpoints: (my_Qsize, my_offset, (edge1, edge2)) of rank `rank`
    (0-based) with 1-based edges; the first mod(nqs, world) ranks take one point more."""
    div, rem = divmod(int(nqs), int(world))
    sizes = [div + (1 if i < rem else 0) for i in range(world)]
    first = sum(sizes[:rank]) + 1
    size = sizes[rank]
    return size, first - 1, (first, first + size - 1)


def partition_by_cost(costs, world: int, rank: int):
    """Contiguous 0-based block [lo, hi) of rank `rank` with the cumulative cost split evenly
    (DistributeQpoints balanced by the work of each q0 instead of by count)."""
    c = np.cumsum(np.asarray(costs, dtype=np.float64))
    tot = c[-1] if len(c) else 0.0
    lo = 0 if rank == 0 else int(np.searchsorted(c, tot * rank / world, side="right"))
    hi = len(c) if rank == world - 1 else int(np.searchsorted(c, tot * (rank + 1) / world, side="right"))
    return lo, hi


def allreduce_linewidths(lw_block, lo: int, hi: int, nq0: int, device=None, group=None):
    """The co_sum of LW_Allq0: this rank's linewidths of q0 in [lo, hi), shape (nT, hi - lo, Ndof),
    zero-padded to (nT, nq0, Ndof) and summed over the ranks.  Returns the full array (numpy)."""
    import torch
    import torch.distributed as dist
    lw_block = np.asarray(lw_block, dtype=np.float64)
    nT, ndof = lw_block.shape[0], lw_block.shape[-1]
    full = torch.zeros((nT, nq0, ndof), dtype=torch.float64, device=device)
    if hi > lo:
        full[:, lo:hi] = torch.from_numpy(np.ascontiguousarray(lw_block[:, : hi - lo])).to(full.device)
    dist.all_reduce(full, op=dist.ReduceOp.SUM, group=group)
    return full.cpu().numpy()


def allgather_blocks(block, lo: int, hi: int, n: int, axis: int = 0, device=None, group=None):
    """Every rank's block [lo, hi) along `axis` of an array of extent n there, gathered into the
    full array on every rank (the per-iteration exchange of F in the iterative solver).  The ranks'
    blocks must tile [0, n) without overlap."""
    import torch
    import torch.distributed as dist
    block = np.asarray(block, dtype=np.float64)
    shape = list(block.shape)
    shape[axis] = n
    full = torch.zeros(shape, dtype=torch.float64, device=device)
    if hi > lo:
        idx = [slice(None)] * len(shape)
        idx[axis] = slice(lo, hi)
        full[tuple(idx)] = torch.from_numpy(np.ascontiguousarray(block)).to(full.device)
    dist.all_reduce(full, op=dist.ReduceOp.SUM, group=group)
    return full.cpu().numpy()
