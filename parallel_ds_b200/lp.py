"""Seeded synthetic LPs (min c^T x, A x <= b, x >= 0) through ds_gen_lp.

Workloads (sizes as the engine's benchmark and tests use them):
  plain_small   m=200,    n=400,    5% density                (CPU-runnable case)
  plain_large   m=50,000, n=100,000, 8 nonzeros per column     (~800k nnz)
  batched       m ~ U{32..512}, n = 2m, 10% density, seed + i
  learned       m=2000,   n=4000,   1% density
  block_angular 32 blocks of 4000 x 8000 (0.1%) + 500 linking rows (0.5%)
"""
import numpy as np

from . import _lib
from ._lib import DsGenSpec, ptr

INF = 1e300
FIXED, FREE, BOXED, UPPER, LOWER = 0, 1, 2, 3, 4


def generate(kind=_lib.GEN_DENSITY, m=200, n=400, density=0.05, per_col=0, seed=0,
             blocks=0, block_m=0, block_n=0, link_rows=0, block_density=0.0, link_density=0.0):
    """Return dict(m, n, row_ptr, col_idx, val, b, c) of a generated LP."""
    L = _lib.lib()
    sp = DsGenSpec(kind, m, n, density, per_col, blocks, block_m, block_n, link_rows,
                   block_density, link_density, seed)
    nnz = L.ds_gen_lp(sp, None, None, None, None, None, 0)
    if nnz < 0:
        raise _lib.DsError(int(nnz), "ds_gen_lp")
    rp = np.zeros(m + 1, np.int32)
    ci = np.zeros(max(nnz, 1), np.int32)
    va = np.zeros(max(nnz, 1), np.float64)
    b = np.zeros(m)
    c = np.zeros(n)
    got = L.ds_gen_lp(sp, ptr(rp, _lib.C.c_int), ptr(ci, _lib.C.c_int), ptr(va, _lib.C.c_double),
                      ptr(b, _lib.C.c_double), ptr(c, _lib.C.c_double), nnz)
    assert got == nnz
    return dict(m=m, n=n, row_ptr=rp, col_idx=ci[:nnz], val=va[:nnz], b=b, c=c, seed=seed)


def plain_small(seed=0):
    return generate(_lib.GEN_DENSITY, 200, 400, density=0.05, seed=seed)


def plain_large(seed=0):
    return generate(_lib.GEN_PER_COL, 50000, 100000, per_col=8, seed=seed)


def learned(seed=0):
    return generate(_lib.GEN_DENSITY, 2000, 4000, density=0.01, seed=seed)


def batched_instance(seed, i, m_lo=32, m_hi=512, density=0.10):
    m = _lib.lib().ds_gen_batch_m(seed, i, m_lo, m_hi)
    return generate(_lib.GEN_DENSITY, m, 2 * m, density=density, seed=seed + i)


def block_angular(seed=0):
    return generate(_lib.GEN_BLOCK, 32 * 4000 + 500, 32 * 8000, blocks=32, block_m=4000, block_n=8000,
                    link_rows=500, block_density=0.001, link_density=0.005, seed=seed)


def typed(lp):
    """The reference's typed form (Problem 8-argument ctor) of A x <= b, x >= 0."""
    m, n = lp["m"], lp["n"]
    return dict(m=m, n=n, row_ptr=lp["row_ptr"], col_idx=lp["col_idx"], val=lp["val"], c=lp["c"],
                col_type=np.full(n, LOWER, np.int32), col_lb=np.zeros(n), col_ub=np.full(n, INF),
                row_type=np.full(m, UPPER, np.int32), row_lb=np.full(m, -INF), row_ub=np.asarray(lp["b"], float))


def to_scipy(lp):
    import scipy.sparse as sp
    return sp.csr_matrix((lp["val"], lp["col_idx"], lp["row_ptr"]), shape=(lp["m"], lp["n"]))
