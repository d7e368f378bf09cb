"""Pair sharding across processes (one process per GPU).

The reference splits pairs round-robin over MPI ranks (pair_id % size ==
rank, lib/correlation_core.cpp:399-409) and rebuilds the matrix with one
MPI_Allreduce(SUM) (:449-457).  Here each rank takes a contiguous,
work-balanced range of the pair list p = a1*(a1-1)/2 + a2 and computes it
with gc_opts.pair_begin/pair_end; a SUM all-reduce over the process group
(NCCL on GPUs, gloo on CPU) rebuilds the off-diagonal entries, and the
diagonal is set to 2000 afterwards (the reference's MPI sum would leave
2000 * size there; pearsify maps either to 1).
"""

from __future__ import annotations

import numpy as np

__all__ = ["pair_shard", "pair_of", "reduce_shards", "sharded_ksg_matrix"]


def pair_shard(npairs: int, rank: int, world: int):
    """Contiguous [begin, end) of the pair list for `rank` (sizes differ by <= 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(npairs, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def pair_of(p: int):
    """(a1, a2) with a2 < a1 of pair index p = a1*(a1-1)/2 + a2."""
    a1 = int((1 + (1 + 8 * p) ** 0.5) // 2)
    while a1 * (a1 - 1) // 2 > p:
        a1 -= 1
    while (a1 + 1) * a1 // 2 <= p:
        a1 += 1
    return a1, p - a1 * (a1 - 1) // 2


def reduce_shards(local: np.ndarray, dist=None) -> np.ndarray:
    """Sum the ranks' shard matrices (each zero outside its shard) and set
    the 2000 diagonal.  `dist` is torch.distributed (or None: one rank)."""
    mat = np.array(local, dtype=np.float64, copy=True)
    np.fill_diagonal(mat, 0.0)
    if dist is not None and dist.is_initialized() and dist.get_world_size() > 1:
        import torch
        backend = dist.get_backend()
        t = torch.from_numpy(mat)
        if backend == "nccl":
            t = t.cuda()
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        mat = t.cpu().numpy()
    np.fill_diagonal(mat, 2000.0)
    return mat


def sharded_ksg_matrix(x, k: int, dist=None, compute=None) -> np.ndarray:
    """KSG MI matrix computed across the process group.

    `compute(x, k, begin, end)` returns the shard matrix; by default the
    GPU entry point gmx_correlation_b200.kraskov_corrmatrix(pairs=...)."""
    n = x.shape[0]
    world = dist.get_world_size() if dist is not None and dist.is_initialized() else 1
    rank = dist.get_rank() if world > 1 else 0
    b, e = pair_shard(n * (n - 1) // 2, rank, world)
    if compute is None:
        from . import kraskov_corrmatrix

        def compute(x_, k_, b_, e_):
            return kraskov_corrmatrix(x_, k_, pairs=(b_, e_))
    return reduce_shards(compute(x, k, b, e), dist)
