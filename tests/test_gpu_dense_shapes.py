"""Dense explicit-inverse mode on shapes that take the strided paths of its
cluster kernels, checked against HiGHS (FP64 optimum oracle), objective
relative error <= 1e-9 and primal feasibility <= 1e-7:

- n above the pivot-row cluster's slot limit (8192): the ticketed k_pivot_row,
  and three slot passes per thread in the dual-update cluster;
- n between 4096 and 8192: two slots per thread in both clusters;
- m above 4096 (dense_max_m raised): two position passes in the CHUZR and
  dual-update clusters.

Each solve also stays on one factorisation as long as the inverse probe
passes, so the test checks the probe-gated rebuilds on these shapes too."""
import numpy as np
import pytest

from conftest import feasibility, highs
from parallel_ds_b200 import _lib
from parallel_ds_b200 import lp as L
from parallel_ds_b200 import solver as S

pytestmark = pytest.mark.gpu


def check(lp, res):
    h = highs(lp)
    assert res["status"] == "optimal" and h.status == 0
    assert abs(res["objective"] - h.fun) <= 1e-9 * max(1.0, abs(h.fun)), (res["objective"], h.fun)
    assert feasibility(lp, res["x"][:lp["n"]]) <= 1e-7


@pytest.mark.parametrize("m,n,density,seed", [(300, 9000, 0.02, 1), (500, 6000, 0.01, 2)])
def test_dense_wide(m, n, density, seed):
    lp = L.generate(_lib.GEN_DENSITY, m, n, density=density, seed=seed)
    res = S.solve_lp(lp, dense_max_m=4096)
    check(lp, res)


def test_dense_tall_above_default_limit():
    lp = L.generate(_lib.GEN_DENSITY, 4150, 4400, density=0.0025, seed=4)
    res = S.solve_lp(lp, dense_max_m=8192)
    check(lp, res)
    assert res["stats"]["iterations"] > 100
