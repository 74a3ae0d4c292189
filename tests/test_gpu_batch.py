"""Batched persistent solver (csrc/batch.cu) against HiGHS (FP64 optimum) and
the oracle (the reference's dual simplex on the CPU).

Tolerances: objective relative error <= 1e-9; primal feasibility
(A x <= b, x >= 0) and dual feasibility (c - A^T y >= 0, y <= 0) <= 1e-7;
statuses equal."""
import numpy as np
import pytest

from conftest import feasibility, highs
from oracle import pyoracle as po
from parallel_ds_b200 import lp as L
from parallel_ds_b200.batch import BatchSolver, to_csc
from parallel_ds_b200._lib import DsError

pytestmark = pytest.mark.gpu


def check_instance(lp, st, z, x, y):
    r = highs(lp)
    assert r.status == 0 and st == 1, (st, r.status)
    assert abs(z - r.fun) <= 1e-9 * max(1.0, abs(r.fun)), (z, r.fun)
    assert feasibility(lp, x) <= 1e-7
    A = L.to_scipy(lp)
    d = lp["c"] - A.T @ y
    assert d.min() >= -1e-7 and y.max() <= 1e-7
    assert abs(lp["c"] @ x - z) <= 1e-9 * max(1.0, abs(z))


@pytest.fixture(scope="module")
def small():
    bs = BatchSolver()
    bs.generate(48, 16, 64, 0.10, seed=7)
    bs.solve()
    return bs


def test_small_batch_matches_highs(small):
    st, obj, it = small.results()
    for i in range(48):
        lp = L.batched_instance(7, i, 16, 64, 0.10)
        x, y = small.solution(i)
        check_instance(lp, st[i], obj[i], x, y)
    assert it.min() > 0


def test_mixed_sizes_match_highs():
    bs = BatchSolver()
    bs.generate(20, 24, 512, 0.10, seed=11)
    bs.solve()
    st, obj, it = bs.results()
    assert bs.stats()["buckets"] >= 3
    for i in range(20):
        lp = L.batched_instance(11, i, 24, 512, 0.10)
        x, y = bs.solution(i)
        check_instance(lp, st[i], obj[i], x, y)


def test_batch_matches_the_oracle(small):
    st, obj, _ = small.results()
    for i in range(0, 48, 6):
        lp = L.batched_instance(7, i, 16, 64, 0.10)
        ref = po.solve_typed(L.typed(lp))
        assert ref["status"] == "optimal" and st[i] == 1
        assert abs(obj[i] - ref["objective"]) <= 1e-9 * max(1.0, abs(ref["objective"]))


def test_schedules_agree_and_runs_are_deterministic():
    bs = BatchSolver()
    bs.generate(40, 16, 160, 0.10, seed=3)
    nb = bs.num_buckets()
    res = []
    for block, g, smem in [(512, 64, 0), (512, 128, 0), (256, 64, 0), (128, 32, 0), (512, 256, 0)]:
        try:
            bs.set_schedule(block, [g] * nb, [smem] * nb)
        except DsError:
            continue                      # does not fit a CTA for the largest bucket
        bs.solve()
        res.append(bs.results())
    bs.tune()
    bs.solve()
    res.append(bs.results())
    assert len(res) >= 3
    st0, ob0, _ = res[0]
    for st, ob, _ in res[1:]:
        np.testing.assert_array_equal(st, st0)
        np.testing.assert_allclose(ob, ob0, rtol=1e-11, atol=1e-11)
    bs.solve()
    st2, ob2, it2 = bs.results()
    np.testing.assert_array_equal(ob2, res[-1][1])
    np.testing.assert_array_equal(it2, res[-1][2])
    assert "g " in bs.stats()["schedule"]


def _lp(A, b, c):
    import scipy.sparse as sp
    A = sp.csr_matrix(np.asarray(A, float))
    return dict(m=A.shape[0], n=A.shape[1], row_ptr=A.indptr.astype(np.int32), col_idx=A.indices.astype(np.int32),
                val=A.data, b=np.asarray(b, float), c=np.asarray(c, float))


def test_statuses_and_edge_instances():
    feasible = _lp([[1, 1], [1, -1]], [4, -1], [1, 2])                 # x1 + x2 <= 4, x1 - x2 <= -1
    infeasible = _lp([[1, 1], [-1, 0]], [-1, 3], [1, 1])               # x1 + x2 <= -1 with x >= 0
    neg_cost = _lp([[1, 1]], [2], [-1, 1])                            # needs phase 1
    one_row = _lp([[-1, 0, 2]], [-0.5], [0.3, 0.0, 1.0])              # a zero-cost column
    empty_col = _lp([[0, -1, 0], [0, 2, 1]], [-1, 5], [1, 1, 1])       # column 0 has no entries
    lps = [feasible, infeasible, neg_cost, one_row, empty_col]
    bs = BatchSolver()
    bs.load(lps)
    bs.solve()
    st, obj, _ = bs.results()
    assert st[0] == 1 and abs(obj[0] - 2.0) <= 1e-12          # x = (0, 1)
    assert st[1] == 2                                          # primal infeasible
    assert st[2] == 5                                          # not dual feasible at the slack basis
    assert st[3] == 1 and abs(obj[3] - 0.15) <= 1e-12         # x1 = 0.5
    assert st[4] == 1 and abs(obj[4] - 1.0) <= 1e-12          # x = (0, 1, 0)
    for i in (0, 1, 3, 4):
        ref = po.solve_typed(L.typed(lps[i]))
        want = {"optimal": 1, "primal_infeasible": 2}[ref["status"]]
        assert st[i] == want
        if want == 1:
            assert abs(obj[i] - ref["objective"]) <= 1e-12


def test_load_rejects_bad_input():
    import ctypes as C
    from parallel_ds_b200._lib import ptr
    bs = BatchSolver()
    big = L.generate(m=1025, n=2050, density=0.001, seed=1)
    with pytest.raises(DsError) as e:
        bs.load([big])
    assert e.value.code == -7                                  # DS_ERR_CAPACITY
    m = np.array([1], np.int32); n = np.array([2], np.int32)
    b = np.array([1.0]); c = np.array([1.0, 1.0]); va = np.array([1.0, 1.0])
    for cp, ri in [([0, 1, 2], [0, 3]),                       # row index beyond m
                   ([1, 1, 2], [0, 0]),                       # pointers not starting at 0
                   ([0, 2, 1], [0, 0])]:                      # decreasing pointers
        cp = np.array(cp, np.int32); ri = np.array(ri, np.int32)
        rc = bs.L.ds_batch_load(bs.h, 1, ptr(m, C.c_int), ptr(n, C.c_int), ptr(cp, C.c_int), ptr(ri, C.c_int),
                                ptr(va, C.c_double), ptr(b, C.c_double), ptr(c, C.c_double))
        assert rc == -1                                        # DS_ERR_ARG


@pytest.mark.parametrize("count,m_lo,m_hi,seed", [(4096, 32, 512, 7000), (65536, 16, 64, 9000)])
def test_full_batched_workloads(count, m_lo, m_hi, seed):
    """The two batched workloads at full size (4096 LPs with m ~ U{32..512};
    65,536 LPs with m ~ U{16..64}; 10% density), autotuned and solved in one
    persistent launch: every status optimal, and 64 instances drawn at random
    checked against HiGHS (objective, primal and dual feasibility)."""
    bs = BatchSolver()
    bs.generate(count, m_lo, m_hi, 0.10, seed=seed)
    bs.tune()
    bs.solve()
    st, obj, it = bs.results()
    assert len(st) == count
    assert np.all(st == 1), np.unique(st, return_counts=True)
    assert it.min() >= 0 and it.mean() > 1     # a few small instances are optimal at the slack basis
    pick = np.random.default_rng(seed).choice(count, size=64, replace=False)
    for i in pick:
        lp = L.batched_instance(seed, int(i), m_lo, m_hi, 0.10)
        x, y = bs.solution(int(i))
        check_instance(lp, st[i], obj[i], x, y)
