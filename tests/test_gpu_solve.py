"""GPU solves through the reference-mirroring interface and the C ABI, checked
against the oracle (same algorithm) and HiGHS (FP64 optimum oracle).

Tolerances: objective relative error <= 1e-9, primal and dual feasibility
<= 1e-7 (statuses must match exactly)."""
import numpy as np
import pytest

from conftest import feasibility, highs, kat_lp
from oracle import pyoracle as po
from parallel_ds_b200 import lp as L
from parallel_ds_b200 import solver as S

pytestmark = pytest.mark.gpu

# Every test runs with the eta file (PFI, the reference's representation) and with
# the explicit dense inverse (the default for m <= 4096).
MODE = {"dense_max_m": 4096}


@pytest.fixture(autouse=True, params=["eta", "dense"])
def linalg_mode(request):
    MODE["dense_max_m"] = 0 if request.param == "eta" else 4096
    yield


def solve_typed_gpu(t, **opts):
    A = S.Matrix(t["val"], t["row_ptr"], t["col_idx"], t["m"], t["n"])
    prob = S.Problem(t["col_type"], t["row_type"], t["c"], t["row_lb"], t["row_ub"], t["col_lb"],
                     t["col_ub"], A)
    prob.transformToComputeForm()
    s = S.CudaDualSimplex(prob, **{**MODE, **opts})
    s.initDualSimplex()
    s.presolve("minInfeas")
    sol = s.solve()
    return s, sol


def test_reference_kats_on_gpu(kats):
    for e in kats["lps"]:
        s, sol = solve_typed_gpu(kat_lp(e), refactor_interval=150, strict_reference=True)
        assert sol.solved and sol.message == "optimal solution", e["name"]
        assert abs(sol.Z - e["z"]) <= e["tol"]
        np.testing.assert_allclose(sol.x[:e["n"]], e["x"][:e["n"]], atol=1e-8)


def test_reference_kat_as_written_hits_limit(kats):
    e = [k for k in kats["lps"] if k["name"] == "Test1"][0]
    s, sol = solve_typed_gpu(kat_lp(e, lower_ub_inf=False), refactor_interval=150,
                             strict_reference=True, max_iterations=500)
    assert s.status() == "iter_limit"


def check_optimal(lp, res, h):
    assert res["status"] == "optimal"
    assert abs(res["objective"] - h.fun) <= 1e-9 * max(1.0, abs(h.fun))
    x = res["x"][:lp["n"]]
    assert feasibility(lp, x) <= 1e-7
    # dual feasibility: structural reduced costs >= -1e-7 at x = 0 (all Lower columns)
    d = res["reduced_costs"]
    assert np.min(d[x <= 1e-9], initial=0.0) >= -1e-7
    # strong duality with the row duals y (y <= 0 for A x <= b)
    y = res["dual"]
    assert np.max(y) <= 1e-7
    assert abs(float(lp["b"] @ y) - h.fun) <= 1e-7 * max(1.0, abs(h.fun))


@pytest.mark.parametrize("seed", range(10))
def test_plain_small_vs_oracle_and_highs(seed):
    lp = L.plain_small(seed)
    res = S.solve_lp(lp, **MODE)
    h = highs(lp)
    check_optimal(lp, res, h)
    orc = po.solve_typed(L.typed(lp))
    assert orc["status"] == "optimal"
    assert abs(res["objective"] - orc["objective"]) <= 1e-9 * abs(orc["objective"])


def test_plain_small_trajectory_matches_oracle():
    """Same algorithm, same pivots: the GPU's (p, q) sequence follows the oracle's
    until the end (both use refactor interval 100)."""
    lp = L.plain_small(0)
    t = L.typed(lp)
    orc = po.solve_typed(t, trace_cap=100000)
    A = S.Matrix(t["val"], t["row_ptr"], t["col_idx"], t["m"], t["n"])
    prob = S.Problem(t["col_type"], t["row_type"], t["c"], t["row_lb"], t["row_ub"], t["col_lb"],
                     t["col_ub"], A)
    s = S.CudaDualSimplex(prob, **MODE)
    s.set_trace(100000)
    s.initDualSimplex()
    s.solve()
    tr = s.trace()
    k = min(len(tr["p"]), len(orc["trace"]["p"]))
    assert k > 50
    same = (tr["p"][:k] == orc["trace"]["p"][:k]) & (tr["q"][:k] == orc["trace"]["q"][:k])
    first_diff = int(np.argmin(same)) if not same.all() else k
    assert first_diff >= min(k, 100), first_diff
    np.testing.assert_allclose(tr["theta"][:first_diff], orc["trace"]["theta"][:first_diff], rtol=1e-9, atol=1e-12)


@pytest.mark.parametrize("seed", range(8))
def test_learned_size_vs_highs(seed):
    lp = L.learned(seed)
    res = S.solve_lp(lp, **MODE)
    check_optimal(lp, res, highs(lp))


def test_status_primal_infeasible():
    from test_oracle import _infeasible_variant
    lp = _infeasible_variant(L.plain_small(1))
    res = S.solve_lp(lp, **MODE)
    assert res["status"] == "primal_infeasible"


def test_status_dual_infeasible():
    from test_oracle import _unbounded_variant
    lp = _unbounded_variant(L.plain_small(2))
    res = S.solve_lp(lp, **MODE)
    assert res["status"] == "dual_infeasible"


def test_phase1_negative_costs_matches_oracle():
    lp = L.plain_small(4)
    lp["c"] = lp["c"] - 0.3
    res = S.solve_lp(lp, **MODE)
    orc = po.solve_typed(L.typed(lp))
    assert res["status"] == orc["status"]
    if orc["status"] == "optimal":
        assert abs(res["objective"] - orc["objective"]) <= 1e-9 * max(1.0, abs(orc["objective"]))
    assert res["stats"]["phase1_iterations"] > 1


def test_load_csr_general_bounds():
    """ds_load_csr with boxed columns and ranged rows (types derived as readMps does)."""
    import ctypes as C
    from parallel_ds_b200._lib import lib, ptr
    rng = np.random.default_rng(3)
    lp = L.plain_small(5)
    m, n = lp["m"], lp["n"]
    col_lb = np.zeros(n); col_ub = np.where(rng.random(n) < 0.3, 0.5, 1e300)
    row_lb = np.where(rng.random(m) < 0.2, lp["b"] - 50.0, -1e300); row_ub = lp["b"].copy()
    from parallel_ds_b200._lib import DsOptions, DsStats
    L_ = lib()
    o = DsOptions()
    L_.ds_default_options(C.byref(o))
    o.dense_max_m = MODE["dense_max_m"]
    h = C.c_void_p()
    assert L_.ds_create(C.byref(o), C.byref(h)) == 0
    try:
        rc = L_.ds_load_csr(h, m, n, ptr(lp["row_ptr"], C.c_int), ptr(lp["col_idx"], C.c_int),
                            ptr(lp["val"], C.c_double), ptr(lp["c"], C.c_double), ptr(col_lb, C.c_double),
                            ptr(col_ub, C.c_double), ptr(row_lb, C.c_double), ptr(row_ub, C.c_double))
        assert rc == 0
        assert L_.ds_solve(h) == 0
        assert L_.ds_get_status(h) == 1
        z = L_.ds_get_objective(h)
        st = DsStats()
        L_.ds_get_stats(h, C.byref(st))
        assert st.bfrt_flips > 0                  # the bound-flipping ratio test was exercised
    finally:
        L_.ds_destroy(h)
    from scipy.optimize import linprog
    A = L.to_scipy(lp)
    import scipy.sparse as sp
    Aub = sp.vstack([A, -A]).tocsr()
    bub = np.concatenate([row_ub, -np.where(row_lb < -1e100, -1e30, row_lb)])
    hs = linprog(lp["c"], A_ub=Aub, b_ub=bub, bounds=list(zip(col_lb, np.where(col_ub > 1e100, None, col_ub))),
                 method="highs-ds")
    assert hs.status == 0
    assert abs(z - hs.fun) <= 1e-9 * max(1.0, abs(hs.fun))
