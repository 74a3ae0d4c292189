"""TEST INFRASTRUCTURE ONLY: ctypes binding of the CPU oracle (libds_oracle.so).

The oracle restates veret-v/parallel_ds's sequential dual simplex
(src/cpu/sequentialDualSimplex.cpp, src/common/baseDualSimplex.tpp).  Only the
tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use it.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libds_oracle.so")

FIXED, FREE, BOXED, UPPER, LOWER = 0, 1, 2, 3, 4
STATUS = {0: "unsolved", 1: "optimal", 2: "primal_infeasible", 3: "dual_infeasible",
          4: "iter_limit", 5: "error"}


class OrOptions(C.Structure):
    _fields_ = [("refactor_interval", C.c_int), ("max_iterations", C.c_int),
                ("strict_reference", C.c_int), ("seed", C.c_ulonglong),
                ("gpu_control_flow", C.c_int), ("verbose", C.c_int), ("var_weight", C.c_void_p),
                ("harris", C.c_int), ("block_lu", C.c_int), ("rt_rel_tol", C.c_double),
                ("col_rel_tol", C.c_double), ("pivot_abs_tol", C.c_double),
                ("shift_costs", C.c_int)]


class OrResult(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("phase1_iterations", C.c_int),
                ("refactors", C.c_int), ("restarts", C.c_int), ("perturbed", C.c_int),
                ("bfrt_flips", C.c_int), ("bump_size", C.c_int),
                ("objective", C.c_double), ("obj_incremental", C.c_double),
                ("min_pivot", C.c_double), ("min_pivot_rel", C.c_double), ("max_step", C.c_double),
                ("refused_pivots", C.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"oracle library missing: {LIB_PATH} (run make -C oracle)")
        _lib = C.CDLL(LIB_PATH)
    return _lib


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct)) if a is not None else None


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def default_options(**kw):
    o = OrOptions()
    lib().or_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def solve_typed(lp, trace_cap=0, **opts):
    """Solve an LP given as a dict with keys m, n, row_ptr, col_idx, val, c,
    col_type, col_lb, col_ub, row_type, row_lb, row_ub.  Returns a dict."""
    m, n = int(lp["m"]), int(lp["n"])
    N = n + m
    o = default_options(**opts)
    r = OrResult()
    x = np.zeros(N); d = np.zeros(N); basis = np.zeros(m, np.int32)
    tp = np.zeros(max(trace_cap, 1), np.int32); tq = np.zeros_like(tp)
    tth = np.zeros(max(trace_cap, 1)); tob = np.zeros_like(tth)
    cnt = C.c_int(0)
    arrs = dict(rp=_i32(lp["row_ptr"]), ci=_i32(lp["col_idx"]), v=_f64(lp["val"]), c=_f64(lp["c"]),
                ct=_i32(lp["col_type"]), cl=_f64(lp["col_lb"]), cu=_f64(lp["col_ub"]),
                rt=_i32(lp["row_type"]), rl=_f64(lp["row_lb"]), ru=_f64(lp["row_ub"]))
    rc = lib().or_solve_typed(
        m, n, _p(arrs["rp"], C.c_int), _p(arrs["ci"], C.c_int), _p(arrs["v"], C.c_double),
        _p(arrs["c"], C.c_double), _p(arrs["ct"], C.c_int), _p(arrs["cl"], C.c_double),
        _p(arrs["cu"], C.c_double), _p(arrs["rt"], C.c_int), _p(arrs["rl"], C.c_double),
        _p(arrs["ru"], C.c_double), C.byref(o), C.byref(r), _p(x, C.c_double), _p(d, C.c_double),
        _p(basis, C.c_int), _p(tp, C.c_int), _p(tq, C.c_int), _p(tth, C.c_double),
        _p(tob, C.c_double), trace_cap, C.byref(cnt))
    if rc != 0:
        raise RuntimeError(f"or_solve_typed returned {rc}")
    k = min(cnt.value, trace_cap)
    return dict(status=STATUS[r.status], status_code=r.status, iterations=r.iterations,
                phase1_iterations=r.phase1_iterations, refactors=r.refactors,
                restarts=r.restarts, perturbed=bool(r.perturbed), bfrt_flips=r.bfrt_flips,
                bump_size=r.bump_size, objective=r.objective, obj_incremental=r.obj_incremental,
                min_pivot=r.min_pivot, min_pivot_rel=r.min_pivot_rel, max_step=r.max_step,
                refused_pivots=r.refused_pivots,
                x=x, d=d, basis=basis, trace_count=cnt.value,
                trace=dict(p=tp[:k].copy(), q=tq[:k].copy(), theta=tth[:k].copy(), obj=tob[:k].copy()))


def dse_pricing(basis, x, lb, ub, typ, beta):
    m = len(basis)
    p, pi, il, pf = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    dl = C.c_double()
    b, xx, l, u, t, be = _i32(basis), _f64(x), _f64(lb), _f64(ub), _i32(typ), _f64(beta)
    lib().or_dse_pricing(m, _p(b, C.c_int), _p(xx, C.c_double), _p(l, C.c_double), _p(u, C.c_double),
                         _p(t, C.c_int), _p(be, C.c_double), C.byref(p), C.byref(pi), C.byref(dl),
                         C.byref(il), C.byref(pf))
    return dict(p=p.value, p_idx=pi.value, delta=dl.value, is_lower=il.value, primal_feasible=pf.value)


def ratio_test(nonbasis, alpha, delta, is_lower, x, d, lb, ub, typ):
    n = len(nonbasis)
    q, qi, nc = C.c_int(), C.c_int(), C.c_int()
    th, do = C.c_double(), C.c_double()
    nb, a, xx, dd, l, u, t = (_i32(nonbasis), _f64(alpha), _f64(x), _f64(d), _f64(lb), _f64(ub), _i32(typ))
    lib().or_ratio_test(n, _p(nb, C.c_int), _p(a, C.c_double), C.c_double(delta), int(is_lower),
                        _p(xx, C.c_double), _p(dd, C.c_double), _p(l, C.c_double), _p(u, C.c_double),
                        _p(t, C.c_int), C.byref(q), C.byref(qi), C.byref(th), C.byref(do), C.byref(nc))
    return dict(q=q.value, q_idx=qi.value, theta=th.value, delta=do.value, num_candidates=nc.value)


def pivot_row(m, n, csc_ptr, csc_row, csc_val, nonbasis, rho):
    out = np.zeros(len(nonbasis))
    cp, cr, cv, nb, r = _i32(csc_ptr), _i32(csc_row), _f64(csc_val), _i32(nonbasis), _f64(rho)
    lib().or_pivot_row(m, n, _p(cp, C.c_int), _p(cr, C.c_int), _p(cv, C.c_double), _p(nb, C.c_int),
                       _p(r, C.c_double), _p(out, C.c_double))
    return out


def pfi_apply(eta, pos, rhs, transpose):
    eta = _f64(eta); pos = _i32(pos); rhs = _f64(rhs)
    T = len(pos); m = len(rhs)
    out = np.zeros(m)
    lib().or_pfi_apply(m, T, _p(eta, C.c_double), _p(pos, C.c_int), _p(rhs, C.c_double),
                       _p(out, C.c_double), int(transpose))
    return out


def dense_solve(n, csr_ptr, csr_col, csr_val, rhs, transpose):
    cp, cc, cv, r = _i32(csr_ptr), _i32(csr_col), _f64(csr_val), _f64(rhs)
    out = np.zeros(n)
    rc = lib().or_dense_solve(n, _p(cp, C.c_int), _p(cc, C.c_int), _p(cv, C.c_double),
                              _p(r, C.c_double), _p(out, C.c_double), int(transpose))
    if rc != 0:
        raise RuntimeError("singular")
    return out
