"""Batched persistent solver: many small LPs  min c^T x, A x <= b, x >= 0  in
one persistent launch (csrc/batch.cu, C ABI ds_batch_*).

    from parallel_ds_b200.batch import BatchSolver
    bs = BatchSolver()
    bs.generate(4096, 32, 512, 0.10, seed=7)   # or bs.load([lp dicts])
    bs.tune()                                  # autotuned schedule (optional)
    bs.solve()
    status, obj, iters = bs.results()

Several GPUs: each rank solves its own instances (seeds offset by
`rank_seed`), no collective in the solve; `gather_results` collects the
per-rank results on every rank afterwards (any torch.distributed backend).
"""
import ctypes as C

import numpy as np

from . import _lib
from ._lib import DsError, ptr

STATUS = _lib.STATUS
MAX_M = 1024


class BatchStats(C.Structure):
    _fields_ = [("count", C.c_int), ("buckets", C.c_int), ("block", C.c_int), ("solve_ms", C.c_double),
                ("tune_ms", C.c_double), ("total_nnz", C.c_longlong), ("schedule", C.c_char * 512)]


def _sig(L):
    IP, DP = C.POINTER(C.c_int), C.POINTER(C.c_double)
    sig = {
        "ds_batch_create": (C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
        "ds_batch_destroy": (C.c_int, [C.c_void_p]),
        "ds_batch_last_error": (C.c_char_p, [C.c_void_p]),
        "ds_batch_load": (C.c_int, [C.c_void_p, C.c_int, IP, IP, IP, IP, DP, DP, DP]),
        "ds_batch_generate": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_ulonglong]),
        "ds_batch_tune": (C.c_int, [C.c_void_p]),
        "ds_batch_gen_arrays": (C.c_longlong, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_ulonglong, IP, IP, IP, IP,
                                               DP, DP, DP, C.POINTER(C.c_longlong)]),
        "ds_batch_set_schedule": (C.c_int, [C.c_void_p, C.c_int, IP, IP, C.c_int]),
        "ds_batch_num_buckets": (C.c_int, [C.c_void_p]),
        "ds_batch_solve": (C.c_int, [C.c_void_p]),
        "ds_batch_get_results": (C.c_int, [C.c_void_p, IP, DP, IP]),
        "ds_batch_get_solution": (C.c_int, [C.c_void_p, C.c_int, DP, DP]),
        "ds_batch_get_stats": (C.c_int, [C.c_void_p, C.POINTER(BatchStats)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def to_csc(lp):
    """(col_ptr, row_idx, val) of a generated LP's A (rows ascending in each column)."""
    m, n = lp["m"], lp["n"]
    rp, ci, va = np.asarray(lp["row_ptr"]), np.asarray(lp["col_idx"]), np.asarray(lp["val"])
    rows = np.repeat(np.arange(m, dtype=np.int32), np.diff(rp))
    order = np.lexsort((rows, ci))
    cp = np.zeros(n + 1, np.int32)
    np.add.at(cp, ci + 1, 1)
    return np.cumsum(cp).astype(np.int32), rows[order].astype(np.int32), va[order].astype(np.float64)


def gen_arrays(count, m_lo, m_hi, density, seed, alloc=None):
    """The ds_batch_load arrays of ds_batch_generate's instances, as a dict
    (m, n, col_ptr, row_idx, val, rhs, cost).  alloc(shape, dtype) makes the
    arrays (e.g. page-locked buffers); default numpy."""
    L = _lib.lib()
    _sig(L)
    alloc = alloc or (lambda shape, dtype: np.zeros(shape, dtype))
    sz = (C.c_longlong * 4)()
    m = alloc(count, np.int32)
    n = alloc(count, np.int32)
    rc = L.ds_batch_gen_arrays(count, m_lo, m_hi, density, seed, ptr(m, C.c_int), ptr(n, C.c_int), None, None,
                               None, None, None, sz)
    if rc != 0:
        raise DsError(int(rc), "ds_batch_gen_arrays")
    out = dict(m=m, n=n, col_ptr=alloc(sz[0], np.int32), row_idx=alloc(sz[1], np.int32),
               val=alloc(sz[1], np.float64), rhs=alloc(sz[2], np.float64), cost=alloc(sz[3], np.float64))
    rc = L.ds_batch_gen_arrays(count, m_lo, m_hi, density, seed, None, None, ptr(out["col_ptr"], C.c_int),
                               ptr(out["row_idx"], C.c_int), ptr(out["val"], C.c_double),
                               ptr(out["rhs"], C.c_double), ptr(out["cost"], C.c_double), sz)
    if rc != 0:
        raise DsError(int(rc), "ds_batch_gen_arrays")
    return out


class BatchSolver:
    """A ds_batch handle on one GPU."""

    def __init__(self, device=0):
        self.L = _lib.lib()
        _sig(self.L)
        self.h = C.c_void_p()
        rc = self.L.ds_batch_create(device, C.byref(self.h))
        if rc != 0:
            raise DsError(rc, "ds_batch_create")
        self.m = self.n = None

    def __del__(self):
        try:
            if self.h:
                self.L.ds_batch_destroy(self.h)
                self.h = C.c_void_p()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != 0:
            msg = self.L.ds_batch_last_error(self.h)
            raise DsError(rc, f"{what}: {msg.decode() if msg else ''}")

    def generate(self, count, m_lo, m_hi, density, seed):
        self._check(self.L.ds_batch_generate(self.h, count, m_lo, m_hi, density, seed), "ds_batch_generate")
        self.m = np.array([self.L.ds_gen_batch_m(seed, i, m_lo, m_hi) for i in range(count)], np.int32)
        self.n = 2 * self.m

    def load(self, lps):
        """Load generated LP dicts (A x <= b, x >= 0)."""
        parts = [to_csc(lp) for lp in lps]
        m = np.array([lp["m"] for lp in lps], np.int32)
        n = np.array([lp["n"] for lp in lps], np.int32)
        cp = np.concatenate([p[0] for p in parts]).astype(np.int32)
        ri = np.concatenate([p[1] for p in parts]).astype(np.int32)
        va = np.concatenate([p[2] for p in parts]).astype(np.float64)
        b = np.concatenate([np.asarray(lp["b"], float) for lp in lps])
        c = np.concatenate([np.asarray(lp["c"], float) for lp in lps])
        self._check(self.L.ds_batch_load(self.h, len(lps), ptr(m, C.c_int), ptr(n, C.c_int), ptr(cp, C.c_int),
                                         ptr(ri, C.c_int), ptr(va, C.c_double), ptr(b, C.c_double),
                                         ptr(c, C.c_double)), "ds_batch_load")
        self.m, self.n = m, n

    def load_arrays(self, a):
        """Load the ds_batch_load arrays of gen_arrays (host buffers, copied)."""
        self._check(self.L.ds_batch_load(self.h, len(a["m"]), ptr(a["m"], C.c_int), ptr(a["n"], C.c_int),
                                         ptr(a["col_ptr"], C.c_int), ptr(a["row_idx"], C.c_int),
                                         ptr(a["val"], C.c_double), ptr(a["rhs"], C.c_double),
                                         ptr(a["cost"], C.c_double)), "ds_batch_load")
        self.m, self.n = np.asarray(a["m"]).copy(), np.asarray(a["n"]).copy()

    def tune(self):
        self._check(self.L.ds_batch_tune(self.h), "ds_batch_tune")

    def num_buckets(self):
        return self.L.ds_batch_num_buckets(self.h)

    def set_schedule(self, block, group_size, binv_in_smem):
        g = np.ascontiguousarray(group_size, np.int32)
        s = np.ascontiguousarray(binv_in_smem, np.int32)
        self._check(self.L.ds_batch_set_schedule(self.h, block, ptr(g, C.c_int), ptr(s, C.c_int), len(g)),
                    "ds_batch_set_schedule")

    def solve(self):
        self._check(self.L.ds_batch_solve(self.h), "ds_batch_solve")

    def results(self):
        k = len(self.m)
        st = np.zeros(k, np.int32)
        obj = np.zeros(k)
        it = np.zeros(k, np.int32)
        self._check(self.L.ds_batch_get_results(self.h, ptr(st, C.c_int), ptr(obj, C.c_double), ptr(it, C.c_int)),
                    "ds_batch_get_results")
        return st, obj, it

    def solution(self, i):
        x = np.zeros(int(self.n[i]))
        y = np.zeros(int(self.m[i]))
        self._check(self.L.ds_batch_get_solution(self.h, i, ptr(x, C.c_double), ptr(y, C.c_double)),
                    "ds_batch_get_solution")
        return x, y

    def stats(self):
        s = BatchStats()
        self._check(self.L.ds_batch_get_stats(self.h, C.byref(s)), "ds_batch_get_stats")
        d = {name: getattr(s, name) for name, _ in s._fields_}
        d["schedule"] = s.schedule.decode()
        return d


# ---------------------------------------------------------------- several GPUs
def rank_seed(seed, rank, count):
    """First instance seed of `rank` when every rank solves `count` instances
    of its own (weak scaling): instance i of rank r is seed + r*count + i."""
    return seed + rank * count


def gather_results(status, objective, iterations, group=None):
    """Concatenate every rank's (status, objective, iterations) in rank order,
    on every rank (torch.distributed.all_gather_object)."""
    import torch.distributed as dist
    mine = (np.asarray(status).tolist(), np.asarray(objective).tolist(), np.asarray(iterations).tolist())
    out = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, mine, group=group)
    st = np.concatenate([np.asarray(o[0], np.int32) for o in out])
    ob = np.concatenate([np.asarray(o[1], np.float64) for o in out])
    it = np.concatenate([np.asarray(o[2], np.int32) for o in out])
    return st, ob, it
