"""Host-side mirror of veret-v/parallel_ds's solver interface over the C ABI.

Same names, argument meaning and call order as the reference's mode-1 path
(src/main.cpp:80-91):

    problem = Problem(bound_type, range_type, costs, lower_range, upper_range,
                      lower_bound, upper_bound, Matrix(val, row_ptr, col_id, m, n))
    problem.transformToComputeForm()
    solver = CudaDualSimplex(problem)
    solver.initDualSimplex()
    solver.presolve("minInfeas")
    solver.solve()
    solution = problem.getSolution()      # LPsolution(Z, solved, x, message)

Errors follow the reference: an LP with more rows than columns raises
"Incorrect constraint size" (problem.tpp:230-239); an unknown presolve method
raises "Unknown phase 1 solver method" (baseDualSimplex.tpp:114-116).
"""
import ctypes as C
from enum import IntEnum

import numpy as np

from . import _lib
from ._lib import DsError, DsOptions, DsStats, ptr

BOUND_INF = 1e100   # problem.hpp:31


class BoundaryType(IntEnum):   # types.hpp:49-57
    Fixed = 0
    Free = 1
    Boxed = 2
    Upper = 3
    Lower = 4


class Matrix:
    """CSR matrix, Matrix(elem_csr, row_ptr, col_id, m, n) (matrix.cpp:21-36)."""

    def __init__(self, elem_csr, row_ptr, col_id, m, n):
        self.val = np.ascontiguousarray(elem_csr, np.float64)
        self.row_ptr = np.ascontiguousarray(row_ptr, np.int32)
        self.col_id = np.ascontiguousarray(col_id, np.int32)
        self.m, self.n = int(m), int(n)

    def getSize(self):
        return (self.m, self.n)


class LPsolution:
    """LPsolution (LPsolution.hpp:22-42)."""

    def __init__(self, Z=0.0, x=None, solved=False, message=""):
        self.Z, self.x, self.solved, self.message = Z, x, solved, message
        self.iterations = 0
        self.phase2_time = 0.0

    def show(self):
        print(f"Z = {self.Z}\nsolved = {self.solved}\nmessage = {self.message}")


MESSAGES = {1: "optimal solution", 2: "dual unbounded", 3: "dual infeasible",
            4: "iteration limit", 5: "error", 0: ""}


class Problem:
    """Problem<Matrix, Vector> 8-argument constructor (problem.tpp:143-173)."""

    def __init__(self, bound_type, range_type, costs, lower_range, upper_range, lower_bound,
                 upper_bound, A):
        m, n = A.getSize()
        if m > n:
            raise RuntimeError("Incorrect constraint size")
        self.A = A
        self.bound_type = np.asarray([int(t) for t in bound_type], np.int32)
        self.range_type = np.asarray([int(t) for t in range_type], np.int32)
        self.costs = np.asarray(costs, np.float64)
        self.lower_range = np.asarray(lower_range, np.float64)
        self.upper_range = np.asarray(upper_range, np.float64)
        self.lower_bound = np.asarray(lower_bound, np.float64)
        self.upper_bound = np.asarray(upper_bound, np.float64)
        self.constraints_size = m
        self.problem_size = n
        self.computational = False
        self._offset = 0.0
        self.solution = LPsolution()

    @classmethod
    def from_bounds(cls, A, c, col_lb, col_ub, row_lb, row_ub):
        """Bound types derived as Problem::readMps does (problem.tpp:350-395)."""
        def kind(lo, hi):
            li, hi_ = abs(lo) > BOUND_INF, abs(hi) > BOUND_INF
            if li and hi_:
                return BoundaryType.Free
            if li:
                return BoundaryType.Upper
            if hi_:
                return BoundaryType.Lower
            return BoundaryType.Fixed if lo == hi else BoundaryType.Boxed
        bt = [kind(a, b) for a, b in zip(col_lb, col_ub)]
        rt = [kind(a, b) for a, b in zip(row_lb, row_ub)]
        return cls(bt, rt, c, row_lb, row_ub, col_lb, col_ub, A)

    @classmethod
    def readMps(cls, filename):
        """Problem::readMps (problem.tpp:332-409) without Clp: the library's MPS
        reader (ds_mps_read) gives the CSR matrix, costs and bounds; bound types
        are derived as readMps does, and the RHS of the objective row becomes the
        offset that getSolution subtracts (problem.tpp:256, 408)."""
        L = _lib.lib()
        path = str(filename).encode()
        m, n, nnz, off = C.c_int(), C.c_int(), C.c_longlong(), C.c_double()
        rc = L.ds_mps_read(path, C.byref(m), C.byref(n), C.byref(nnz), None, None, None, None, None, None, None,
                           None, C.byref(off))
        if rc != 0:
            raise DsError(rc, L.ds_mps_last_error().decode())
        m, n, nnz = m.value, n.value, nnz.value
        rp = np.zeros(m + 1, np.int32)
        ci = np.zeros(max(nnz, 1), np.int32)
        va = np.zeros(max(nnz, 1))
        c, clb, cub, rlb, rub = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(m), np.zeros(m)
        rc = L.ds_mps_read(path, C.byref(C.c_int()), C.byref(C.c_int()), C.byref(C.c_longlong()),
                           ptr(rp, C.c_int), ptr(ci, C.c_int), ptr(va, C.c_double), ptr(c, C.c_double),
                           ptr(clb, C.c_double), ptr(cub, C.c_double), ptr(rlb, C.c_double), ptr(rub, C.c_double),
                           C.byref(off))
        if rc != 0:
            raise DsError(rc, L.ds_mps_last_error().decode())
        p = cls.from_bounds(Matrix(va[:nnz], rp, ci[:nnz], m, n), c, clb, cub, rlb, rub)
        p._offset = off.value
        return p

    def transformToComputeForm(self):
        """Slack columns are appended inside the engine (problem.tpp:176-226)."""
        self.computational = True

    def checkWellScaled(self):
        """Problem::checkWellScaled (problem.tpp:26-43): log10(max|a| / min|a|) < 2
        over the stored nonzeros (False for an empty matrix, as there)."""
        a = np.abs(self.A.val)
        if a.size == 0:
            return False
        with np.errstate(divide="ignore", invalid="ignore"):
            return bool(np.log10(a.max() / a.min()) < 2)

    def scale(self):
        """Problem::scale (problem.tpp:46-103): each row divided by its largest
        |a| (row bounds too), then each column by its largest |a| after that;
        costs are divided and column bounds multiplied by the column factors, so
        x_scaled = scale_cols * x.  getSolution maps x back and re-prices it with
        the original costs.  The reference leaves scaling off (problem.tpp:396-400);
        an empty row keeps factor 1 here (the reference would read past the row)."""
        A = self.A
        m, n = A.getSize()
        val = A.val.copy()
        rows = np.repeat(np.arange(m), np.diff(A.row_ptr))
        self.scale_rows = np.ones(m)
        amax = np.zeros(m)
        np.maximum.at(amax, rows, np.abs(val))
        nz = np.diff(A.row_ptr) > 0
        self.scale_rows[nz] = amax[nz]
        val = val / self.scale_rows[rows]
        self.lower_range = self.lower_range / self.scale_rows
        self.upper_range = self.upper_range / self.scale_rows
        self.scale_cols = np.zeros(n)
        np.maximum.at(self.scale_cols, A.col_id, np.abs(val))
        sc = self.scale_cols[A.col_id]
        val = np.where(sc != 0, val / np.where(sc != 0, sc, 1.0), val)
        has = self.scale_cols != 0
        safe = np.where(has, self.scale_cols, 1.0)
        self.costs = np.where(has, self.costs / safe, self.costs)
        self.upper_bound = np.where(has, self.upper_bound * safe, self.upper_bound)
        self.lower_bound = np.where(has, self.lower_bound * safe, self.lower_bound)
        self.A = Matrix(val, A.row_ptr, A.col_id, m, n)
        self.scaled = True

    def getSolution(self):
        """Problem::getSolution (problem.tpp:241-259): unscale the structurals and
        re-price them with the original costs when scaled, then subtract the
        objective offset."""
        if getattr(self, "scaled", False):
            n = self.A.n
            has = self.scale_cols != 0
            safe = np.where(has, self.scale_cols, 1.0)
            x = np.asarray(self.solution.x, np.float64).copy()
            x[:n] = np.where(has, x[:n] / safe, x[:n])
            self.solution.x = x
            self.solution.Z = float(np.where(has, self.costs * safe, self.costs) @ x[:n])
        self.solution.Z -= self._offset
        return self.solution


class CudaDualSimplex:
    """CudaDualSimplex (cudaDualSimplex.hpp:27-92) backed by libds_b200.so."""

    def __init__(self, problem, refactor_interval=100, max_iterations=2000000, pricing="dse",
                 strict_reference=False, seed=12345, device=0, learned_margin=0.5, learned_mix=0.05,
                 learned_pdhg_iters=4000, dense_max_m=4096, dense_refactor_interval=400,
                 learned_start_iteration=-1, pdhg_cluster=1, model=None, verbose=0, factor="sparse"):
        self.problem = problem
        self.L = _lib.lib()
        o = DsOptions()
        self.L.ds_default_options(C.byref(o))
        o.refactor_interval = refactor_interval
        o.max_iterations = max_iterations
        o.pricing = _lib.PRICING_LEARNED if pricing == "learned" else _lib.PRICING_DSE
        o.strict_reference = int(bool(strict_reference))
        o.seed = seed
        o.device = device
        o.learned_margin = learned_margin
        o.learned_mix = learned_mix
        o.learned_pdhg_iters = learned_pdhg_iters
        o.dense_max_m = dense_max_m
        o.dense_refactor_interval = dense_refactor_interval
        o.learned_start_iteration = learned_start_iteration
        o.pdhg_cluster = pdhg_cluster
        if factor not in ("sparse", "dense"):
            raise ValueError(f"unknown factorisation {factor!r}")
        o.factor_mode = _lib.FACTOR_DENSE if factor == "dense" else _lib.FACTOR_SPARSE
        o.verbose = verbose
        self.opts = o
        self.h = C.c_void_p()
        rc = self.L.ds_create(C.byref(o), C.byref(self.h))
        if rc != 0:
            raise DsError(rc, "ds_create")
        self.model = model
        self.loaded = False
        self.presolved = False

    def __del__(self):
        try:
            if self.h:
                self.L.ds_destroy(self.h)
                self.h = C.c_void_p()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != 0:
            msg = self.L.ds_last_error(self.h)
            raise DsError(rc, f"{what}: {msg.decode() if msg else ''}")

    def initDualSimplex(self):
        p = self.problem
        A = p.A
        self._arrs = (A.row_ptr, A.col_id, A.val, p.costs, p.bound_type, p.lower_bound, p.upper_bound,
                      p.range_type, p.lower_range, p.upper_range)
        rc = self.L.ds_load_typed(self.h, A.m, A.n, ptr(A.row_ptr, C.c_int), ptr(A.col_id, C.c_int),
                                  ptr(A.val, C.c_double), ptr(p.costs, C.c_double),
                                  ptr(p.bound_type, C.c_int), ptr(p.lower_bound, C.c_double),
                                  ptr(p.upper_bound, C.c_double), ptr(p.range_type, C.c_int),
                                  ptr(p.lower_range, C.c_double), ptr(p.upper_range, C.c_double))
        self._check(rc, "ds_load_typed")
        if self.model is not None:
            self.model.attach(self)
        self.loaded = True

    def presolve(self, presolver_method_name="minInfeas"):
        if presolver_method_name != "minInfeas":
            raise RuntimeError("Unknown phase 1 solver method")
        self.presolved = True   # phase 1 runs inside ds_solve, as presolve does before solve()

    def solve(self):
        if not self.loaded:
            self.initDualSimplex()
        rc = self.L.ds_solve(self.h)
        self._check(rc, "ds_solve")
        st = self.L.ds_get_status(self.h)
        n, m = self.problem.A.n, self.problem.A.m
        x = np.zeros(n)
        s = np.zeros(m)
        self.L.ds_get_primal(self.h, ptr(x, C.c_double), ptr(s, C.c_double))
        sol = self.problem.solution
        sol.Z = self.L.ds_get_objective(self.h)
        sol.x = np.concatenate([x, s])
        sol.solved = st == 1
        sol.message = MESSAGES.get(st, "")
        sol.iterations = self.L.ds_get_iterations(self.h)
        sol.phase2_time = self.stats()["solve_ms"]
        return sol

    # ---- queries the reference does not expose
    def status(self):
        return _lib.STATUS[self.L.ds_get_status(self.h)]

    def dual(self):
        y = np.zeros(self.problem.A.m)
        self._check(self.L.ds_get_dual(self.h, ptr(y, C.c_double)), "ds_get_dual")
        return y

    def reduced_costs(self):
        d = np.zeros(self.problem.A.n)
        self._check(self.L.ds_get_reduced_costs(self.h, ptr(d, C.c_double)), "ds_get_reduced_costs")
        return d

    def basis(self):
        b = np.zeros(self.problem.A.m, np.int32)
        self._check(self.L.ds_get_basis(self.h, ptr(b, C.c_int)), "ds_get_basis")
        return b

    def stats(self):
        st = DsStats()
        self.L.ds_get_stats(self.h, C.byref(st))
        return st.as_dict()

    def set_trace(self, cap):
        self._check(self.L.ds_set_trace(self.h, int(cap)), "ds_set_trace")

    def trace(self):
        cap = 1 << 22
        cnt = C.c_int(0)
        self.L.ds_get_trace(self.h, None, None, None, None, C.byref(cnt))
        k = cnt.value
        p = np.zeros(k, np.int32); q = np.zeros(k, np.int32)
        th = np.zeros(k); ob = np.zeros(k)
        self.L.ds_get_trace(self.h, ptr(p, C.c_int), ptr(q, C.c_int), ptr(th, C.c_double),
                            ptr(ob, C.c_double), C.byref(cnt))
        del cap
        return dict(p=p, q=q, theta=th, obj=ob)

    def pdhg_estimate(self, iters):
        """PDHG estimate (x [n], row duals y [m]) of the loaded LP after `iters` iterations."""
        if not self.loaded:
            self.initDualSimplex()
        x = np.zeros(self.problem.A.n)
        y = np.zeros(self.problem.A.m)
        self._check(self.L.ds_pdhg_estimate(self.h, int(iters), ptr(x, C.c_double), ptr(y, C.c_double)),
                    "ds_pdhg_estimate")
        return x, y

    def set_feature_trace(self, every, cap):
        """Record candidate-row features every `every` phase-2 iterations (training data)."""
        self._check(self.L.ds_set_feature_trace(self.h, int(every), int(cap)), "ds_set_feature_trace")

    def feature_trace(self):
        """(features [k x 12] float32, meta [k x 3] (iteration, position, variable), total seen)."""
        cnt, tot = C.c_int(0), C.c_int(0)
        self._check(self.L.ds_get_feature_trace(self.h, None, None, C.byref(cnt), C.byref(tot)),
                    "ds_get_feature_trace")
        k = cnt.value
        F = np.zeros((k, _lib.NUM_FEATURES), np.float32)
        M = np.zeros((k, 3), np.int32)
        self._check(self.L.ds_get_feature_trace(self.h, ptr(F, C.c_float), ptr(M, C.c_int), C.byref(cnt),
                                                C.byref(tot)), "ds_get_feature_trace")
        return F, M, tot.value


def problem_from_lp(lp):
    """Problem (reference 8-argument form) of a generated LP dict (lp.generate)."""
    from .lp import typed
    t = typed(lp)
    A = Matrix(t["val"], t["row_ptr"], t["col_idx"], t["m"], t["n"])
    prob = Problem(t["col_type"], t["row_type"], t["c"], t["row_lb"], t["row_ub"], t["col_lb"],
                   t["col_ub"], A)
    prob.transformToComputeForm()
    return prob


def solve_lp(lp, **opts):
    """Solve a generated LP dict (lp.generate) and return a result dict."""
    s = CudaDualSimplex(problem_from_lp(lp), **opts)
    s.initDualSimplex()
    s.presolve("minInfeas")
    sol = s.solve()
    out = dict(status=s.status(), objective=sol.Z, x=sol.x, iterations=sol.iterations,
               stats=s.stats(), dual=s.dual(), reduced_costs=s.reduced_costs(), basis=s.basis())
    return out
