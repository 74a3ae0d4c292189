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
