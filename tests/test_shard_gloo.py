"""Multi-rank pair sharding on CPU: two gloo ranks each compute their shard
(through the oracle, standing in for the GPU shard) and the all-reduce
rebuilds the reference's full matrix."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from gmx_correlation_b200.shard import pair_of, pair_shard, reduce_shards, sharded_ksg_matrix


def test_pair_shard_partition():
    for npairs in (1, 7, 2016, 30381):
        for world in (1, 2, 3, 8):
            spans = [pair_shard(npairs, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == npairs
            assert all(spans[r][1] == spans[r + 1][0] for r in range(world - 1))
            sizes = [e - b for b, e in spans]
            assert max(sizes) - min(sizes) <= 1


def test_pair_of_roundtrip():
    for p in range(5000):
        a1, a2 = pair_of(p)
        assert 0 <= a2 < a1 and a1 * (a1 - 1) // 2 + a2 == p


def _oracle_shard(x, k, b, e):
    from oracle import Oracle
    o = Oracle()
    X, psi = o.prepare(x)
    n = x.shape[0]
    m = np.zeros((n, n))
    np.fill_diagonal(m, 2000.0)
    for p in range(b, e):
        a1, a2 = pair_of(p)
        mi = o.ksg_pair_detail(X, psi, k, a1, a2)["mi"]
        m[a1, a2] = m[a2, a1] = mi
    return m


def _worker(rank, world, port, x, k, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mat = sharded_ksg_matrix(x, k, dist, compute=_oracle_shard)
        out[rank] = mat
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_rebuild_the_reference_matrix(oracle, world):
    """Each rank computes its shard; the all-gather of the packed pair values
    (uneven shards with three ranks: 36 pairs) rebuilds the reference's matrix
    on every rank."""
    from gmx_correlation_b200.synth import synth_traj
    x = synth_traj(9, 160, 4, 0.08, seed=77)
    k = 6
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, x, k, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    want = oracle.ksg_matrix(x, k)
    for r in range(world):
        np.testing.assert_array_equal(out[r], want)


def test_pairs_to_matrix_layout():
    from gmx_correlation_b200.shard import pairs_to_matrix
    n = 7
    v = np.arange(n * (n - 1) // 2, dtype=float) + 1.0
    m = pairs_to_matrix(v, n)
    for p in range(len(v)):
        a1, a2 = pair_of(p)
        assert m[a1, a2] == m[a2, a1] == v[p]
    assert np.all(np.diag(m) == 2000.0)


def test_single_rank_reduce_is_identity():
    m = np.arange(16, dtype=float).reshape(4, 4)
    r = reduce_shards(m, None)
    assert np.all(np.diag(r) == 2000.0)
    off = ~np.eye(4, dtype=bool)
    np.testing.assert_array_equal(r[off], m[off])
