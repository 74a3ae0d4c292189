"""Failure paths, made on the host (no GPU fault, trap or hang is provoked):
non-finite input, singular bases handed to ds_basis_solve, an eta-file
capacity request above the limit.  Each ends with an error code, and the
handle stays usable afterwards.

The reference has no checks for these (cudaSparseMatrix.cpp:124,130 exit the
process; addEtaMatrix, PFIfactor.cpp:40-74, has no overflow guard); the
engine reports DS_ERR_ARG / DS_ERR_NUMERIC instead."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from parallel_ds_b200 import _lib
from parallel_ds_b200 import lp as L
from parallel_ds_b200._lib import DsOptions, lib, ptr

pytestmark = pytest.mark.gpu

DS_ERR_ARG, DS_ERR_NUMERIC = -1, -5


def make(opts=None):
    L_ = lib()
    h = C.c_void_p()
    o = DsOptions()
    L_.ds_default_options(C.byref(o))
    for k, v in (opts or {}).items():
        setattr(o, k, v)
    rc = L_.ds_create(C.byref(o), C.byref(h))
    return rc, h


def load(h, t):
    L_ = lib()
    return L_.ds_load_typed(h, t["m"], t["n"], ptr(t["row_ptr"], C.c_int), ptr(t["col_idx"], C.c_int),
                            ptr(t["val"], C.c_double), ptr(t["c"], C.c_double), ptr(t["col_type"], C.c_int),
                            ptr(t["col_lb"], C.c_double), ptr(t["col_ub"], C.c_double),
                            ptr(t["row_type"], C.c_int), ptr(t["row_lb"], C.c_double), ptr(t["row_ub"], C.c_double))


@pytest.mark.parametrize("where", ["cost", "matrix", "row_bound", "col_bound"])
def test_nan_input_rejected_then_handle_usable(where):
    L_ = lib()
    rc, h = make()
    assert rc == 0
    try:
        good = L.typed(L.plain_small(0))
        bad = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in good.items()}
        key = {"cost": "c", "matrix": "val", "row_bound": "row_ub", "col_bound": "col_lb"}[where]
        bad[key][3] = np.nan
        assert load(h, bad) == DS_ERR_ARG
        assert b"finite" in L_.ds_last_error(h) or b"NaN" in L_.ds_last_error(h)
        assert load(h, good) == 0
        assert L_.ds_solve(h) == 0 and L_.ds_get_status(h) == 1
    finally:
        L_.ds_destroy(h)


def test_infinite_matrix_entry_rejected():
    L_ = lib()
    rc, h = make()
    try:
        t = L.typed(L.plain_small(1))
        t = dict(t, val=t["val"].copy())
        t["val"][0] = np.inf
        assert load(h, t) == DS_ERR_ARG
    finally:
        L_.ds_destroy(h)


def test_refactor_interval_above_eta_capacity_rejected():
    rc, _ = make({"refactor_interval": 201})
    assert rc == DS_ERR_ARG
    rc, _ = make({"refactor_interval": 0})
    assert rc == DS_ERR_ARG


def _singular_lp():
    """plain_small(0) with columns 0 and 1 replaced by the same column
    (entries 1 and 2 in rows 0 and 1, exact in binary arithmetic), and
    column 2 emptied except in row 5."""
    lp = L.plain_small(0)
    A = L.to_scipy(lp).tolil()
    for j in (0, 1, 2):
        A[:, j] = 0.0
    for j in (0, 1):
        A[0, j] = 1.0
        A[1, j] = 2.0
    A[5, 2] = 1.5
    A = sp.csr_matrix(A)
    A.eliminate_zeros()
    A.sort_indices()
    return dict(lp, row_ptr=A.indptr.astype(np.int32), col_idx=A.indices.astype(np.int32), val=A.data)


@pytest.mark.parametrize("mode", ["sparse", "eta_gj", "dense"])
@pytest.mark.parametrize("case", ["numeric", "structural"])
def test_singular_basis_reported(mode, case):
    L_ = lib()
    opts = {} if mode == "dense" else {"dense_max_m": 0, "factor_mode": _lib.FACTOR_DENSE if mode == "eta_gj"
                                       else _lib.FACTOR_SPARSE}
    rc, h = make(opts)
    assert rc == 0
    try:
        lp = _singular_lp()
        t = L.typed(lp)
        assert load(h, t) == 0
        m, n = lp["m"], lp["n"]
        if case == "numeric":      # columns 0 and 1 are equal; rows 0 and 1 are the bump's rows
            basis = np.array([0, 1] + [n + r for r in range(2, m)], np.int32)
        else:                      # column 2 has no entry in the bump's rows (0 and 1)
            basis = np.array([0, 2] + [n + r for r in range(2, m)], np.int32)
        rhs = np.ones(m)
        out = np.zeros(m)
        rc = L_.ds_basis_solve(h, ptr(basis, C.c_int), ptr(rhs, C.c_double), ptr(out, C.c_double), 1, 0)
        assert rc == DS_ERR_NUMERIC, rc
        assert b"singular" in L_.ds_last_error(h)
        # the handle still solves with a nonsingular basis
        good = np.array([0] + [n + r for r in range(1, m)], np.int32)
        rc = L_.ds_basis_solve(h, ptr(good, C.c_int), ptr(rhs, C.c_double), ptr(out, C.c_double), 1, 0)
        assert rc == 0
        assert abs(out[0] - 1.0) < 1e-15          # x_0 = rhs_0 / A[0, 0]
    finally:
        L_.ds_destroy(h)


def test_scorer_wait_timeout_falls_back_to_dse():
    """The scorer's bounded MMA-completion wait, made to run out by a one-poll
    bound (ds_model_set_wait_limit): ds_solve returns DS_ERR_DEVICE_WAIT, the
    timed-out iterations fall back to DSE pricing, and the solve still ends
    optimal at the plain solve's objective.  With the default bound restored
    the same handles solve cleanly."""
    from parallel_ds_b200 import learned as LN
    from parallel_ds_b200 import solver as S
    from parallel_ds_b200._lib import DsError
    L_ = lib()
    lp = L.learned(2001)
    plain = S.solve_lp(lp, pricing="dse")
    model = LN.LeavingRowScorer.load()
    assert L_.ds_model_set_wait_limit(model.h, 1) == 0
    s = S.CudaDualSimplex(S.problem_from_lp(lp), pricing="learned", model=model)
    s.initDualSimplex()
    with pytest.raises(DsError) as ei:
        s.solve()
    assert ei.value.code == -6                         # DS_ERR_DEVICE_WAIT
    assert s.status() == "optimal"
    z = L_.ds_get_objective(s.h)
    assert abs(z - plain["objective"]) <= 1e-9 * max(1.0, abs(plain["objective"]))
    assert s.stats()["learned_fallback"] > 0
    assert L_.ds_model_set_wait_limit(model.h, 0) == 0
    s2 = S.CudaDualSimplex(S.problem_from_lp(lp), pricing="learned", model=model)
    s2.initDualSimplex()
    sol = s2.solve()
    assert s2.status() == "optimal"
    assert abs(sol.Z - plain["objective"]) <= 1e-9 * max(1.0, abs(plain["objective"]))
