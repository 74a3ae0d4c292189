"""GPU parity of single kernels against the oracle on identical input vectors.

Index selection (CHUZR pricing, CHUZC ratio test with bound flipping) and the
pivot-row values are bit-exact; the PFI eta apply uses a different (one-pass)
summation and is compared with a relative tolerance of 1e-12.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import pyoracle as po
from parallel_ds_b200._lib import lib, ptr

pytestmark = pytest.mark.gpu

IP, DP = C.c_int, C.c_double


def gpu_dse(basis, x, lb, ub, typ, beta):
    m, N = len(basis), len(x)
    p, pi, il, pf = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    dl = C.c_double()
    arr = [np.ascontiguousarray(a, t) for a, t in ((basis, np.int32), (x, float), (lb, float), (ub, float),
                                                  (typ, np.int32), (beta, float))]
    rc = lib().ds_kernel_dse_pricing(m, N, ptr(arr[0], IP), ptr(arr[1], DP), ptr(arr[2], DP), ptr(arr[3], DP),
                                     ptr(arr[4], IP), ptr(arr[5], DP), C.byref(p), C.byref(pi), C.byref(dl),
                                     C.byref(il), C.byref(pf))
    assert rc == 0
    return dict(p=p.value, p_idx=pi.value, delta=dl.value, is_lower=il.value, primal_feasible=pf.value)


def gpu_ratio(nonbasis, alpha, delta, is_lower, x, d, lb, ub, typ):
    n, N = len(nonbasis), len(x)
    q, qi, nc = C.c_int(), C.c_int(), C.c_int()
    th, do = C.c_double(), C.c_double()
    a = [np.ascontiguousarray(v, t) for v, t in ((nonbasis, np.int32), (alpha, float), (x, float), (d, float),
                                                (lb, float), (ub, float), (typ, np.int32))]
    rc = lib().ds_kernel_ratio_test(n, N, ptr(a[0], IP), ptr(a[1], DP), delta, int(is_lower), ptr(a[2], DP),
                                    ptr(a[3], DP), ptr(a[4], DP), ptr(a[5], DP), ptr(a[6], IP), C.byref(q),
                                    C.byref(qi), C.byref(th), C.byref(do), C.byref(nc))
    assert rc == 0
    return dict(q=q.value, q_idx=qi.value, theta=th.value, delta=do.value, num_candidates=nc.value)


def random_state(rng, m, n, infeas_frac=0.3):
    N = n + m
    typ = rng.choice([0, 1, 2, 3, 4], size=N, p=[0.1, 0.05, 0.25, 0.2, 0.4]).astype(np.int32)
    lb = np.where(rng.random(N) < 0.5, 0.0, rng.standard_normal(N))
    ub = lb + rng.random(N) * 3
    lb[typ == 0] = ub[typ == 0] = rng.standard_normal((typ == 0).sum())
    ub[typ == 4] = 1e300
    lb[typ == 3] = -1e300
    x = np.where(rng.random(N) < 0.5, lb, ub)
    x = np.where(np.abs(x) > 1e100, 0.0, x)
    bad = rng.random(N) < infeas_frac
    x[bad] += rng.standard_normal(bad.sum()) * 2
    tiny = rng.random(N) < 0.05
    x[tiny] = lb[tiny] - rng.choice([5e-11, 2e-9, 3e-8], tiny.sum())
    x = np.where(np.abs(x) > 1e100, 0.0, x)
    return typ, lb, ub, x


@pytest.mark.parametrize("seed", range(12))
def test_dse_pricing_bit_exact(seed):
    rng = np.random.default_rng(seed)
    m = int(rng.integers(1, 3000)); n = int(rng.integers(m, 2 * m + 2))
    typ, lb, ub, x = random_state(rng, m, n)
    basis = rng.permutation(n + m)[:m].astype(np.int32)
    beta = rng.random(m) * 4 + 1e-3
    if seed % 3 == 0:   # exact weight ties: first index must win
        dup = rng.integers(0, m, size=min(m, 20))
        beta[dup] = 1.0
        x[basis[dup]] = lb[basis[dup]] - 0.5
        typ[basis[dup]] = 4
    a = po.dse_pricing(basis, x, lb, ub, typ, beta)
    b = gpu_dse(basis, x, lb, ub, typ, beta)
    assert a == b


def test_dse_pricing_feasible_and_empty():
    m, n = 50, 60
    typ = np.full(n + m, 4, np.int32)
    lb = np.zeros(n + m); ub = np.full(n + m, 1e300); x = np.ones(n + m)
    basis = np.arange(n, n + m, dtype=np.int32)
    beta = np.ones(m)
    a = po.dse_pricing(basis, x, lb, ub, typ, beta)
    b = gpu_dse(basis, x, lb, ub, typ, beta)
    assert a == b and b["primal_feasible"] == 1 and b["p"] == -1


@pytest.mark.parametrize("seed", range(6))
def test_pivot_row_bit_exact(seed):
    rng = np.random.default_rng(100 + seed)
    m = int(rng.integers(1, 4000)); n = int(rng.integers(m, 3 * m))
    dens = min(1.0, 20.0 / m)
    import scipy.sparse as sp
    A = sp.random(m, n, density=dens, random_state=seed, format="csc", data_rvs=rng.standard_normal)
    A.sort_indices()
    nonbasis = rng.permutation(n + m)[:n].astype(np.int32)
    rho = rng.standard_normal(m)
    rho[rng.random(m) < 0.3] = 0.0
    ref = po.pivot_row(m, n, A.indptr, A.indices, A.data, nonbasis, rho)
    got = np.zeros(n)
    a = [np.ascontiguousarray(v, t) for v, t in ((A.indptr, np.int32), (A.indices, np.int32), (A.data, float),
                                                (nonbasis, np.int32), (rho, float))]
    assert lib().ds_kernel_pivot_row(m, n, ptr(a[0], IP), ptr(a[1], IP), ptr(a[2], DP), ptr(a[3], IP),
                                     ptr(a[4], DP), ptr(got, DP)) == 0
    np.testing.assert_array_equal(got, ref)


@pytest.mark.parametrize("seed", range(12))
def test_ratio_test_bit_exact(seed):
    rng = np.random.default_rng(200 + seed)
    m = int(rng.integers(1, 1500)); n = int(rng.integers(m, 3 * m + 3))
    typ, lb, ub, x = random_state(rng, m, n, infeas_frac=0.0)
    nonbasis = rng.permutation(n + m)[:n].astype(np.int32)
    alpha = rng.standard_normal(n) * (rng.random(n) < 0.6)
    alpha[rng.random(n) < 0.05] = 3e-6          # |alpha| <= EPS_A band
    d = np.abs(rng.standard_normal(n + m))
    if seed % 2 == 0:                            # degenerate: many d_j == 0 -> theta ties at 0
        d[rng.random(n + m) < 0.4] = 0.0
    if seed % 3 == 0:                            # ties within EPS_Z
        d = np.round(d, 1)
    delta = float(rng.standard_normal() * 3)
    is_lower = int(delta < 0)
    a = po.ratio_test(nonbasis, alpha, delta, is_lower, x, d, lb, ub, typ)
    b = gpu_ratio(nonbasis, alpha, delta, is_lower, x, d, lb, ub, typ)
    assert a == b


def test_ratio_test_bfrt_flips():
    """All-boxed candidates: the bound-flipping loop passes several breakpoints."""
    n, m = 40, 10
    N = n + m
    typ = np.full(N, 2, np.int32); lb = np.zeros(N); ub = np.full(N, 0.1)
    x = lb.copy()
    nonbasis = np.arange(n, dtype=np.int32)
    alpha = np.linspace(0.5, 2.0, n)
    d = np.linspace(0.01, 0.4, N)
    for delta in (0.05, 0.3, 1.0, 5.0, 100.0):
        a = po.ratio_test(nonbasis, alpha, delta, 0, x, d, lb, ub, typ)
        b = gpu_ratio(nonbasis, alpha, delta, 0, x, d, lb, ub, typ)
        assert a == b, delta


@pytest.mark.parametrize("transpose", [0, 1])
def test_pfi_apply(transpose):
    rng = np.random.default_rng(7)
    m, T = 3000, 60
    eta = rng.standard_normal((T, m)) * (rng.random((T, m)) < 0.2)
    pos = rng.integers(0, m, T).astype(np.int32)
    pos[5] = pos[4]                       # repeated pivot position
    for t in range(T):
        eta[t, pos[t]] = 1.0 / (1.0 + rng.random())
    rhs = rng.standard_normal(m)
    ref = po.pfi_apply(eta, pos, rhs, transpose)
    got = np.zeros(m)
    e = np.ascontiguousarray(eta); p = np.ascontiguousarray(pos)
    assert lib().ds_kernel_pfi_apply(m, T, ptr(e, DP), ptr(p, IP), ptr(rhs, DP), ptr(got, DP), transpose) == 0
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
