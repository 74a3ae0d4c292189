"""Same-box per-kernel baseline: the reference's own GPU kernels, built for
sm_100a from its source (oracle/_ref/librefkern.so, see oracle/Makefile), timed
against the engine's replacements on identical inputs of the large eta-file
workload's size (m = 50,000, n = 100,000, 8 nonzeros per column).

  pivot row  spmvUpdateTKernel (cudaKernels.cu:108-157)  vs k_pivot_row
  eta file   etaSolveKernel    (cudaKernels.cu:266-322)  vs the engine's
             chain solve + streaming pass (FTRAN) / chain solve (BTRAN)

Our results are checked against numpy (the reference kernels are only timed:
spmvUpdateTKernel's gather reads other blocks' partial sums without a grid
barrier, and etaSolveKernel's forward step reads y[p] while the thread owning p
overwrites it, so their outputs are not a reliable check).  Times: the engine's
kernels are bracketed by CUDA events inside ds_kernel_* (ds_kernel_last_time,
minimum of five calls); the reference's by events around 20 back-to-back
launches after 3 warm-up launches (mean)."""
import ctypes as C
import os

import numpy as np
import pytest

from parallel_ds_b200 import lp as L
from parallel_ds_b200._lib import lib, ptr

pytestmark = pytest.mark.gpu

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "librefkern.so")


@pytest.fixture(scope="module")
def refk():
    if not os.path.exists(REF):
        pytest.skip("oracle/_ref/librefkern.so not built (needs the reference sources)")
    R = C.CDLL(REF)
    IP, DP, FP = C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_float)
    R.rk_pivot_row.argtypes = [C.c_int, C.c_int, IP, IP, DP, DP, IP, C.c_int, DP, C.c_int, C.c_int, FP]
    R.rk_eta_solve.argtypes = [C.c_int, C.c_int, DP, IP, DP, C.c_int, DP, C.c_int, C.c_int, FP]
    return R


def ours_ms(call):
    L_ = lib()
    best = None
    for _ in range(5):
        assert call() == 0
        ms = C.c_double()
        assert L_.ds_kernel_last_time(C.byref(ms)) == 0
        best = ms.value if best is None else min(best, ms.value)
    return best


@pytest.fixture(scope="module")
def large():
    return L.plain_large(0)


def test_pivot_row_vs_reference_kernel(refk, large):
    lp = large
    m, n = lp["m"], lp["n"]
    A = L.to_scipy(lp).tocsc()
    A.sort_indices()
    rng = np.random.default_rng(0)
    rho = rng.standard_normal(m)
    N = n + m
    nonbasis = np.sort(rng.choice(N, size=n, replace=False)).astype(np.int32)
    cp, cr, cv = A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float64)
    alpha = np.zeros(n)
    t_ours = ours_ms(lambda: lib().ds_kernel_pivot_row(m, n, ptr(cp, C.c_int), ptr(cr, C.c_int), ptr(cv, C.c_double),
                                                       ptr(nonbasis, C.c_int), ptr(rho, C.c_double),
                                                       ptr(alpha, C.c_double)))
    full = np.concatenate([A.T @ rho, rho])
    ref = full[nonbasis]
    assert np.max(np.abs(alpha - ref)) <= 1e-12 * (1 + np.max(np.abs(ref)))
    # [A | I] by columns for the reference kernel
    import scipy.sparse as sp
    AI = sp.hstack([A, sp.identity(m, format="csc")]).tocsc()
    AI.sort_indices()
    out = np.zeros(n)
    ms = C.c_float()
    rc = refk.rk_pivot_row(m, N, ptr(AI.indptr.astype(np.int32), C.c_int), ptr(AI.indices.astype(np.int32), C.c_int),
                           ptr(AI.data.astype(np.float64), C.c_double), ptr(rho, C.c_double),
                           ptr(nonbasis, C.c_int), n, ptr(out, C.c_double), 3, 20, C.byref(ms))
    assert rc == 0
    print(f"\n[kernel baseline] pivot row m={m} n={n}: k_pivot_row {t_ours * 1e3:.1f} us, "
          f"reference spmvUpdateTKernel {ms.value * 1e3:.1f} us ({ms.value / t_ours:.2f}x)")
    assert t_ours < ms.value


def pfi_forward(eta, pos, x):
    y = x.copy()
    for t in range(len(pos)):
        a = y[pos[t]]
        y += a * eta[t]
        y[pos[t]] = a * eta[t][pos[t]]
    return y


def pfi_backward(eta, pos, x):
    y = x.copy()
    for t in range(len(pos) - 1, -1, -1):
        y[pos[t]] = eta[t] @ y
    return y


@pytest.mark.parametrize("transpose", [0, 1])
def test_eta_file_vs_reference_kernel(refk, transpose):
    m, T = 50000, 50
    rng = np.random.default_rng(1 + transpose)
    pos = rng.choice(m, size=T, replace=False).astype(np.int32)
    eta = rng.standard_normal((T, m)) * 1e-2
    for t in range(T):
        eta[t, pos[t]] = 1.0 + rng.random()          # pivot entries 1/alpha_p away from zero
    x = rng.standard_normal(m)
    sol = np.zeros(m)
    e = np.ascontiguousarray(eta)
    t_ours = ours_ms(lambda: lib().ds_kernel_pfi_apply(m, T, ptr(e, C.c_double), ptr(pos, C.c_int),
                                                       ptr(x, C.c_double), ptr(sol, C.c_double), transpose))
    ref = (pfi_backward if transpose else pfi_forward)(eta, pos, x)
    assert np.max(np.abs(sol - ref)) <= 1e-11 * (1 + np.max(np.abs(ref)))
    y = np.zeros(m)
    ms = C.c_float()
    assert refk.rk_eta_solve(m, T, ptr(e, C.c_double), ptr(pos, C.c_int), ptr(x, C.c_double), transpose,
                             ptr(y, C.c_double), 3, 20, C.byref(ms)) == 0
    print(f"\n[kernel baseline] eta file m={m} T={T} {'BTRAN' if transpose else 'FTRAN'}: engine "
          f"{t_ours * 1e3:.1f} us, reference etaSolveKernel {ms.value * 1e3:.1f} us ({ms.value / t_ours:.2f}x)")
    assert t_ours < ms.value
