"""Problem.scale / checkWellScaled / getSolution on the CPU (problem.tpp:26-103,
241-259): the scaled arrays worked out by hand, and the CPU oracle solving a
scaled LP to the unscaled optimum once getSolution maps it back."""
import numpy as np

from oracle import pyoracle as po
from parallel_ds_b200 import lp as L
from parallel_ds_b200 import solver as S

INF = 1e300


def small():
    A = S.Matrix([2.0, 4.0, 1.0, 8.0], [0, 2, 4], [0, 1, 0, 1], 2, 2)
    return S.Problem.from_bounds(A, [3.0, 5.0], [0.0, 1.0], [10.0, INF], [-INF, 2.0], [12.0, 16.0])


def test_scale_by_hand():
    p = small()
    assert p.checkWellScaled()          # log10(8 / 1) < 2
    p.scale()
    # rows / (4, 8) -> [[.5, 1], [.125, 1]]; columns / (.5, 1)
    np.testing.assert_array_equal(p.A.val, [1.0, 1.0, 0.25, 1.0])
    np.testing.assert_array_equal(p.scale_rows, [4.0, 8.0])
    np.testing.assert_array_equal(p.scale_cols, [0.5, 1.0])
    np.testing.assert_array_equal(p.costs, [6.0, 5.0])
    np.testing.assert_array_equal(p.lower_bound, [0.0, 1.0])
    np.testing.assert_array_equal(p.upper_bound, [5.0, INF])
    np.testing.assert_array_equal(p.lower_range, [-INF / 4, 0.25])
    np.testing.assert_array_equal(p.upper_range, [3.0, 2.0])


def test_well_scaled_threshold():
    A = S.Matrix([1.0, 150.0], [0, 2], [0, 1], 1, 2)
    assert not S.Problem.from_bounds(A, [1, 1], [0, 0], [INF, INF], [-INF], [1.0]).checkWellScaled()
    assert not S.Problem.from_bounds(S.Matrix([], [0, 0], [], 1, 2), [1, 1], [0, 0], [INF, INF], [-INF],
                                     [1.0]).checkWellScaled()


def typed(p):
    return dict(m=p.A.m, n=p.A.n, row_ptr=p.A.row_ptr, col_idx=p.A.col_id, val=p.A.val, c=p.costs,
                col_type=p.bound_type, col_lb=p.lower_bound, col_ub=p.upper_bound,
                row_type=p.range_type, row_lb=p.lower_range, row_ub=p.upper_range)


def badly_scaled(seed):
    """A generated LP with rows and columns multiplied by factors over six decades."""
    lp = L.plain_small(seed)
    m, n = lp["m"], lp["n"]
    r = np.random.default_rng(seed)
    rs, cs = 10.0 ** r.uniform(-3, 3, m), 10.0 ** r.uniform(-3, 3, n)
    rows = np.repeat(np.arange(m), np.diff(lp["row_ptr"]))
    val = lp["val"] * rs[rows] * cs[lp["col_idx"]]
    A = S.Matrix(val, lp["row_ptr"], lp["col_idx"], m, n)
    # x_new = x / cs: costs c * cs, rows b * rs
    return S.Problem.from_bounds(A, lp["c"] * cs, np.zeros(n), np.full(n, INF), np.full(m, -INF), lp["b"] * rs)


def test_scaled_solve_maps_back_to_the_unscaled_optimum():
    p0 = badly_scaled(1)
    assert not p0.checkWellScaled()
    r0 = po.solve_typed(typed(p0))
    p1 = badly_scaled(1)
    p1.scale()
    assert p1.checkWellScaled() or np.abs(p1.A.val).max() <= 1.0
    r1 = po.solve_typed(typed(p1))
    assert r0["status"] == r1["status"] == "optimal"
    p1.solution = S.LPsolution(r1["objective"], np.asarray(r1["x"], float), True, "optimal solution")
    sol = p1.getSolution()
    assert abs(sol.Z - r0["objective"]) <= 1e-9 * max(1.0, abs(r0["objective"]))
    np.testing.assert_allclose(sol.x[:p1.A.n], np.asarray(r0["x"])[:p1.A.n], rtol=1e-7, atol=1e-9)
