"""CPU tests of the oracle: pinned against the reference's own known answers and
against HiGHS (scipy) as the FP64 optimum oracle."""
import numpy as np
import pytest

from conftest import feasibility, highs, kat_lp
from oracle import pyoracle as po
from parallel_ds_b200 import lp as L


def test_reference_lp_kats(kats):
    """tests/simple_tests_DS.cpp:12-145: analytic optima (and x) of four LPs."""
    for e in kats["lps"]:
        r = po.solve_typed(kat_lp(e), refactor_interval=150, strict_reference=1)
        assert r["status"] == "optimal", e["name"]
        assert abs(r["objective"] - e["z"]) <= e["tol"], (e["name"], r["objective"], e["z"])
        np.testing.assert_allclose(r["x"][:e["n"]], e["x"][:e["n"]], atol=1e-8)


def test_reference_kats_as_written_loop(kats):
    """With upper_bound = 0 on Lower columns, exactly as the reference test source
    writes them, checkVarIsInfeas' case fallthrough (baseDualSimplex.tpp:447-453)
    reads the 0 as an upper bound and the reference never terminates.  Test3
    reaches optimality before pricing ever runs."""
    for e in kats["lps"]:
        r = po.solve_typed(kat_lp(e, lower_ub_inf=False), refactor_interval=150,
                           strict_reference=1, max_iterations=3000)
        if e["name"] == "Test3":
            assert r["status"] == "optimal"
        else:
            assert r["status"] == "iter_limit", e["name"]


def test_reference_lu_kats(kats):
    """tests/test_math.cpp:12-49: 3x3 solves, transposed and not."""
    for k in kats["lu"]:
        sol = po.dense_solve(3, k["row_ptr"], k["col_idx"], k["val"], k["rhs"], k["transpose"])
        np.testing.assert_allclose(sol, k["expected"], rtol=0, atol=1e-15)


@pytest.mark.parametrize("seed", range(8))
def test_plain_small_matches_highs(seed):
    lp = L.plain_small(seed)
    r = po.solve_typed(L.typed(lp))
    h = highs(lp)
    assert r["status"] == "optimal"
    assert abs(r["objective"] - h.fun) <= 1e-9 * abs(h.fun)
    assert feasibility(lp, r["x"][:lp["n"]]) <= 1e-7


def test_strict_and_guarded_agree_on_plain():
    lp = L.plain_small(3)
    a = po.solve_typed(L.typed(lp), strict_reference=1)
    b = po.solve_typed(L.typed(lp), strict_reference=0)
    assert a["status"] == b["status"] == "optimal"
    assert a["iterations"] == b["iterations"]


def _infeasible_variant(lp):
    """A row with all-nonnegative coefficients and b < 0 (no x >= 0 satisfies it)."""
    lp = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in lp.items()}
    r = 0
    s, e = lp["row_ptr"][r], lp["row_ptr"][r + 1]
    lp["val"][s:e] = np.abs(lp["val"][s:e]) + 0.1
    lp["b"][r] = -1.0
    return lp


def _unbounded_variant(lp):
    """A column with all-nonpositive coefficients and negative cost: an improving ray."""
    lp = {k: (v.copy() if isinstance(v, np.ndarray) else v) for k, v in lp.items()}
    j = 0
    mask = lp["col_idx"] == j
    lp["val"][mask] = -np.abs(lp["val"][mask]) - 0.1
    lp["c"][j] = -1.0
    return lp


def test_status_infeasible():
    lp = _infeasible_variant(L.plain_small(1))
    r = po.solve_typed(L.typed(lp))
    assert r["status"] == "primal_infeasible"
    assert highs(lp).status == 2


def test_status_unbounded():
    lp = _unbounded_variant(L.plain_small(2))
    r = po.solve_typed(L.typed(lp))
    assert r["status"] == "dual_infeasible"
    assert highs(lp).status == 3


def test_phase1_negative_costs():
    """c with negative entries: the slack basis is not dual feasible, phase 1 runs."""
    lp = L.plain_small(4)
    lp["c"] = lp["c"] - 0.3
    r = po.solve_typed(L.typed(lp))
    h = highs(lp)
    assert r["phase1_iterations"] > 1
    if h.status == 0:
        assert r["status"] == "optimal"
        assert abs(r["objective"] - h.fun) <= 1e-9 * max(1.0, abs(h.fun))
    else:
        assert r["status"] in ("dual_infeasible", "primal_infeasible")


def test_pfi_apply_matches_eta_products():
    """linalg::PFIsolve (linalg.cpp:12-46) against explicit eta matrices."""
    rng = np.random.default_rng(0)
    m, T = 12, 5
    eta = rng.standard_normal((T, m))
    pos = rng.integers(0, m, T).astype(np.int32)
    rhs = rng.standard_normal(m)
    E = []
    for t in range(T):
        Et = np.eye(m)
        Et[:, pos[t]] = eta[t]     # inverse eta matrix: column p replaced by eta
        E.append(Et)
    fwd = rhs.copy()
    for t in range(T):
        fwd = E[t] @ fwd
    np.testing.assert_allclose(po.pfi_apply(eta, pos, rhs, 0), fwd, rtol=1e-12, atol=1e-12)
    bwd = rhs.copy()
    for t in reversed(range(T)):
        bwd = E[t].T @ bwd
    np.testing.assert_allclose(po.pfi_apply(eta, pos, rhs, 1), bwd, rtol=1e-12, atol=1e-12)


def test_ratio_test_tie_rule():
    """simpleRatioTest (tpp:546-572): strict '<', ties within EPS_Z prefer larger |alpha|."""
    n, m = 4, 1
    N = n + m
    nonbasis = np.arange(n, dtype=np.int32)
    x = np.zeros(N); lb = np.zeros(N); ub = np.full(N, 1e300)
    typ = np.full(N, 4, np.int32)
    alpha = np.array([1.0, 2.0, 4.0, 3.0])
    d = np.array([1.0, 2.0, 4.0 + 1e-11 * 4, 3.0])   # theta = 1, 1, 1 + 1e-11, 1
    r = po.ratio_test(nonbasis, alpha, 0.5, 0, x, d, lb, ub, typ)
    # 0 taken (theta 1), 1 by tie (|alpha| 2 > 1), 2 by tie (theta drifts to
    # 1 + 1e-11, |alpha| 4), then 3 by the strict '<' (1 < 1 + 1e-11)
    assert r["q_idx"] == 3 and r["num_candidates"] == 4
    d2 = d.copy(); d2[3] = 3.0 * (1 + 1e-11)      # now 3 ties with 2 but |alpha| 3 < 4
    assert po.ratio_test(nonbasis, alpha, 0.5, 0, x, d2, lb, ub, typ)["q_idx"] == 2


def test_oracle_pivot_statistics():
    """The oracle's numerical diagnostics: the smallest phase-2 pivot |alpha_q[p]|
    (absolute and relative to its column) and the largest primal step."""
    r = po.solve_typed(L.typed(L.plain_small(3)))
    assert r["status"] == "optimal"
    assert 0 < r["min_pivot_rel"] <= 1.0
    assert r["min_pivot"] > 1e-5 * 0.999        # the ratio test only takes |alpha| > EPS_A
    assert 0 < r["max_step"] < 1e12


@pytest.mark.parametrize("block_lu", [1, 2])
def test_oracle_block_factorisation(block_lu):
    """The oracle's experimental factorisations of the structural block
    (singleton triangularisation + dense or Markowitz kernel LU) reach HiGHS's
    optimum like its default dense LU."""
    from parallel_ds_b200 import _lib
    for lp in (L.plain_small(1), L.generate(_lib.GEN_PER_COL, 600, 1200, per_col=8, seed=2)):
        h = highs(lp)
        r = po.solve_typed(L.typed(lp), block_lu=block_lu)
        assert r["status"] == "optimal"
        assert abs(r["objective"] - h.fun) <= 1e-9 * max(1.0, abs(h.fun))


def test_oracle_stabilised_rules_reach_highs_optimum():
    """The oracle's experimental stabilisation for large LPs (pivot tolerance
    1e-2 in the ratio test, cost shifting instead of phase 1 once the costs are
    perturbed, block-triangular LU) on a 3000 x 6000 LP of the large workload's
    generator: HiGHS's optimum, with hardly any phase 1."""
    from parallel_ds_b200 import _lib
    lp = L.generate(_lib.GEN_PER_COL, 3000, 6000, per_col=8, seed=0)
    r = po.solve_typed(L.typed(lp), block_lu=2, pivot_abs_tol=1e-2, shift_costs=1)
    h = highs(lp)
    assert r["status"] == "optimal"
    assert abs(r["objective"] - h.fun) <= 1e-9 * max(1.0, abs(h.fun))
    assert r["phase1_iterations"] < 100
    assert r["min_pivot"] >= 1e-2 * 0.5


def test_oracle_column_relative_pivot_refusal():
    """The oracle's experimental refusal of a pivot that is small against its own
    FTRAN column (|alpha_q[p]| < col_rel_tol * max|alpha_q|): the row is blocked
    for a while, the basis refactorised, and the solve still ends at HiGHS's
    optimum, with every pivot taken above the bar."""
    from parallel_ds_b200 import _lib
    lp = L.generate(_lib.GEN_PER_COL, 600, 1200, per_col=8, seed=2)
    r = po.solve_typed(L.typed(lp), col_rel_tol=1e-3)
    h = highs(lp)
    assert r["status"] == "optimal"
    assert abs(r["objective"] - h.fun) <= 1e-9 * max(1.0, abs(h.fun))
    assert r["refused_pivots"] > 0
    assert r["min_pivot_rel"] >= 1e-3
