"""Pair sharding across processes (one process per GPU).

The reference splits pairs round-robin over MPI ranks (pair_id % size ==
rank, lib/correlation_core.cpp:399-409) and rebuilds the matrix with one
MPI_Allreduce(SUM) of the n x n matrix (:449-457).  Here each rank takes a
contiguous, work-balanced range of the pair list p = a1*(a1-1)/2 + a2 and
computes it with gc_opts.pair_begin/pair_end; one all-gather of the packed
pair values (8 bytes per pair, NCCL on GPUs, gloo on CPU) gives every rank
the whole list, from which the matrix is assembled with the 2000 diagonal.
reduce_shards keeps the reference's sum-of-matrices form.
"""

from __future__ import annotations

import numpy as np

__all__ = ["pair_shard", "pair_of", "reduce_shards", "gather_pairs", "pairs_to_matrix", "sharded_ksg_matrix"]


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


def gather_pairs(local, npairs: int, dist=None):
    """All-gather of the ranks' packed shard values (rank r holds pairs
    pair_shard(npairs, r, world)): every rank gets the whole packed list.
    `local` is a 1-D float64 array or torch tensor (on the GPU for NCCL);
    the shards are padded to one length for the collective.  Returns a
    tensor on local's device (a numpy array for numpy input)."""
    import torch
    as_numpy = isinstance(local, np.ndarray)
    t = torch.from_numpy(local) if as_numpy else local
    world = dist.get_world_size() if dist is not None and dist.is_initialized() else 1
    if world == 1:
        return local
    width = -(-npairs // world)
    pad = torch.zeros(width, dtype=torch.float64, device=t.device)
    pad[: t.numel()] = t
    out = torch.empty(world * width, dtype=torch.float64, device=t.device)
    dist.all_gather_into_tensor(out, pad)
    parts = [out[r * width: r * width + (pair_shard(npairs, r, world)[1] - pair_shard(npairs, r, world)[0])]
             for r in range(world)]
    full = torch.cat(parts)
    return full.cpu().numpy() if as_numpy else full


def pairs_to_matrix(values, n: int) -> np.ndarray:
    """n x n matrix of packed pair values (p = a1*(a1-1)/2 + a2): both
    triangles and the 2000 diagonal, as kraskov_corrmatrix writes it."""
    v = np.asarray(values, dtype=np.float64)
    m = np.zeros((n, n))
    a1, a2 = np.tril_indices(n, -1)
    order = np.argsort(a1 * (a1 - 1) // 2 + a2, kind="stable")
    m[a1[order], a2[order]] = v
    m[a2[order], a1[order]] = v
    np.fill_diagonal(m, 2000.0)
    return m


def sharded_ksg_matrix(x, k: int, dist=None, compute=None) -> np.ndarray:
    """KSG MI matrix computed across the process group.

    `compute(x, k, begin, end)` returns the shard matrix (zero outside the
    shard); by default the GPU entry point
    gmx_correlation_b200.kraskov_corrmatrix(pairs=...).  The shards' packed
    values are all-gathered (gather_pairs) and the matrix assembled."""
    n = x.shape[0]
    npairs = n * (n - 1) // 2
    world = dist.get_world_size() if dist is not None and dist.is_initialized() else 1
    rank = dist.get_rank() if world > 1 else 0
    b, e = pair_shard(npairs, rank, world)
    if compute is None:
        from . import kraskov_corrmatrix

        def compute(x_, k_, b_, e_):
            return kraskov_corrmatrix(x_, k_, pairs=(b_, e_))
    shard = compute(x, k, b, e)
    a1, a2 = np.tril_indices(n, -1)
    p = a1 * (a1 - 1) // 2 + a2
    sel = (p >= b) & (p < e)
    local = np.zeros(e - b)
    local[p[sel] - b] = shard[a1[sel], a2[sel]]
    if world > 1 and dist.get_backend() == "nccl":
        import torch
        full = gather_pairs(torch.from_numpy(local).cuda(), npairs, dist).cpu().numpy()
    else:
        full = gather_pairs(local, npairs, dist)
    return pairs_to_matrix(full, n)
