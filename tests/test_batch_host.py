"""Host side of the batched path on the CPU: CSC conversion, the weak-scaling
seed split and the cross-rank gather of results (world size 2, gloo)."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from parallel_ds_b200 import lp as L
from parallel_ds_b200.batch import gather_results, rank_seed, to_csc


def test_to_csc_matches_scipy():
    lp = L.batched_instance(5, 3, 16, 64, 0.10)
    cp, ri, va = to_csc(lp)
    A = L.to_scipy(lp).tocsc()
    A.sort_indices()
    np.testing.assert_array_equal(cp, A.indptr)
    np.testing.assert_array_equal(ri, A.indices)
    np.testing.assert_array_equal(va, A.data)


def test_rank_seeds_partition_instances():
    count, world, seed = 100, 4, 7
    seen = [rank_seed(seed, r, count) + i for r in range(world) for i in range(count)]
    assert len(set(seen)) == world * count and min(seen) == seed


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    k = 3 + rank                                   # ragged shards
    st = np.full(k, 1 + rank, np.int32)
    ob = np.arange(k, dtype=np.float64) + 10 * rank
    it = np.arange(k, dtype=np.int32) * (rank + 1)
    gs, go, gi = gather_results(st, ob, it)
    if rank == 0:
        np.save(out, np.stack([gs.astype(float), go, gi.astype(float)]))
    dist.barrier()
    dist.destroy_process_group()


def test_gather_results_two_ranks(tmp_path):
    out = str(tmp_path / "g.npy")
    port = 29500 + os.getpid() % 2000
    mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
    g = np.load(out)
    np.testing.assert_array_equal(g[0], [1, 1, 1, 2, 2, 2, 2])
    np.testing.assert_array_equal(g[1], [0, 1, 2, 10, 11, 12, 13])
    np.testing.assert_array_equal(g[2], [0, 1, 2, 0, 2, 4, 6])


STATUS_CODE = {"optimal": 1, "primal_infeasible": 2, "dual_infeasible": 3, "iter_limit": 4, "error": 5}


def _solve_shard(seed, first, count, m_lo=16, m_hi=48):
    """Solve instances first .. first+count-1 of the batched generator on the
    CPU oracle: (status codes, objectives, iterations)."""
    from oracle import pyoracle as po
    st, ob, it = [], [], []
    for i in range(first, first + count):
        lp = L.batched_instance(seed, i, m_lo, m_hi, 0.10)
        r = po.solve_typed(L.typed(lp))
        st.append(STATUS_CODE[r["status"]]); ob.append(r["objective"]); it.append(r["iterations"])
    return np.array(st, np.int32), np.array(ob), np.array(it, np.int32)


def _shard_worker(rank, world, port, count, seed, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    first = rank_seed(seed, rank, count) - seed      # instance index of this rank's first LP
    st, ob, it = _solve_shard(seed, first, count)
    gs, go, gi = gather_results(st, ob, it)
    if rank == 0:
        np.save(out, np.stack([gs.astype(float), go, gi.astype(float)]))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_batch_union_equals_single_rank(tmp_path):
    """Weak-scaling shards of the batched workload over two gloo ranks (each
    rank solves its own instance range, no collective in the solve): the
    gathered results equal one rank solving the union."""
    out = str(tmp_path / "s.npy")
    port = 31500 + os.getpid() % 2000
    count, seed = 6, 11
    mp.spawn(_shard_worker, args=(2, port, count, seed, out), nprocs=2, join=True)
    g = np.load(out)
    st, ob, it = _solve_shard(seed, 0, 2 * count)
    np.testing.assert_array_equal(g[0], st)
    np.testing.assert_array_equal(g[1], ob)
    np.testing.assert_array_equal(g[2], it)
    assert np.all(st == 1)
