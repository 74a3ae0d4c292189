"""Eta-file solves through the sparse LU of the basis's structural block, on
LPs whose bumps run to thousands of columns: the large eta-file workload's
generator (8 nonzeros per column at uniform random rows, N(0,1) values) at
m = 3000 and 4000, checked against HiGHS.

Tolerances: objective relative error <= 1e-9, primal and dual feasibility
<= 1e-7, status optimal."""
import numpy as np
import pytest

from conftest import feasibility, highs
from parallel_ds_b200 import _lib
from parallel_ds_b200 import lp as L
from parallel_ds_b200 import solver as S

pytestmark = pytest.mark.gpu


def per_col_lp(seed, m=10000):
    return L.generate(_lib.GEN_PER_COL, m, 2 * m, per_col=8, seed=seed)


@pytest.mark.parametrize("seed,m", [(0, 3000), (1, 4000)])
def test_per_col_vs_highs(seed, m):
    lp = per_col_lp(seed, m)
    res = S.solve_lp(lp, dense_max_m=0)
    h = highs(lp)
    assert res["status"] == "optimal"
    assert abs(res["objective"] - h.fun) <= 1e-9 * max(1.0, abs(h.fun)), (res["objective"], h.fun)
    x = res["x"][:lp["n"]]
    assert feasibility(lp, x) <= 1e-7
    d = res["reduced_costs"]
    assert np.min(d[x <= 1e-9], initial=0.0) >= -1e-7
    y = res["dual"]
    assert np.max(y) <= 1e-7
    assert abs(float(lp["b"] @ y) - h.fun) <= 1e-7 * max(1.0, abs(h.fun))
    st = res["stats"]
    assert st["bump_size"] > 500 and st["lu_kernel"] > 0 and st["lu_levels"] > 0, st


def test_sparse_and_gauss_jordan_factors_agree():
    """The same eta-file solve with the sparse LU and with the Gauss-Jordan
    inverse of the bump: same status and objective (the pivot sequences may
    part where rounding differs, the optimum may not)."""
    lp = per_col_lp(3, m=2000)
    a = S.solve_lp(lp, dense_max_m=0, factor="sparse")
    b = S.solve_lp(lp, dense_max_m=0, factor="dense")
    assert a["status"] == b["status"] == "optimal"
    assert abs(a["objective"] - b["objective"]) <= 1e-9 * max(1.0, abs(b["objective"]))


@pytest.mark.parametrize("dense_max_m", [0, 4096])
def test_block_angular_scaled_vs_highs(dense_max_m):
    """The block-angular workload's structure at a scale the test suite can
    afford: 8 diagonal blocks of 400 x 800 (4 nonzeros per block column, as
    the 4000 x 8000 blocks at 0.1% have) plus 50 linking rows over all
    columns at 0.5%; eta-file mode (sparse LU) and dense mode."""
    lp = L.generate(_lib.GEN_BLOCK, 8 * 400 + 50, 8 * 800, blocks=8, block_m=400, block_n=800, link_rows=50,
                    block_density=0.01, link_density=0.005, seed=4)
    res = S.solve_lp(lp, dense_max_m=dense_max_m)
    h = highs(lp)
    assert res["status"] == "optimal"
    assert abs(res["objective"] - h.fun) <= 1e-9 * max(1.0, abs(h.fun)), (res["objective"], h.fun)
    assert feasibility(lp, res["x"][:lp["n"]]) <= 1e-7
