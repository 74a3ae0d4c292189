"""MPS input on the GPU: ds_load_mps through the C ABI and Problem.readMps
through the reference-mirroring interface (src/main.cpp:80-91 with
problem.readMps), against HiGHS and against the same LP loaded from arrays."""
import ctypes as C

import numpy as np
import pytest

from test_mps import FREE1, FREE2, FREE3, SAMPLE, SAMPLE_SOLVE, highs_general, to_mps, typed, write
from oracle import pyoracle as po
from parallel_ds_b200 import _lib
from parallel_ds_b200 import lp as L
from parallel_ds_b200 import solver as S

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("text", [SAMPLE_SOLVE, SAMPLE])
def test_readmps_mirror_path(tmp_path, text):
    """problem.readMps -> transformToComputeForm -> CudaDualSimplex -> getSolution:
    the reported objective is c^T x minus the file's objective offset (SAMPLE has
    a free column, which the solver's crash makes basic)."""
    f = write(tmp_path, text)
    problem = S.Problem.readMps(f)
    problem.transformToComputeForm()
    solver = S.CudaDualSimplex(problem)
    solver.initDualSimplex()
    solver.presolve("minInfeas")
    solver.solve()
    sol = problem.getSolution()
    h = highs_general(S.Problem.readMps(f))
    assert sol.solved and sol.message == "optimal solution"
    assert abs(sol.Z - (h.fun - (-3.5))) <= 1e-9 * max(1.0, abs(h.fun))


def test_load_mps_c_abi(tmp_path):
    lib = _lib.lib()
    o = _lib.DsOptions()
    lib.ds_default_options(C.byref(o))
    h = C.c_void_p()
    assert lib.ds_create(C.byref(o), C.byref(h)) == 0
    try:
        off = C.c_double()
        assert lib.ds_load_mps(h, str(write(tmp_path, SAMPLE_SOLVE)).encode(), C.byref(off)) == 0
        assert off.value == -3.5
        assert lib.ds_solve(h) == 0
        assert lib.ds_get_status(h) == 1
        assert abs(lib.ds_get_objective(h) - (-5.5)) <= 1e-9 * 5.5
        rc = lib.ds_load_mps(h, str(tmp_path / "absent.mps").encode(), None)
        assert rc == -1 and b"cannot open" in lib.ds_mps_last_error()
    finally:
        lib.ds_destroy(h)


def test_mps_round_trip_solves_identically(tmp_path):
    """An LP written to MPS and read back loads the same arrays, so the GPU solve
    takes the same pivots to the same objective, bit for bit."""
    lp = L.plain_small(1)
    a = S.solve_lp(lp)
    p = S.Problem.readMps(write(tmp_path, to_mps(lp)))
    s = S.CudaDualSimplex(p)
    s.initDualSimplex()
    s.presolve("minInfeas")
    sol = s.solve()
    assert s.status() == a["status"] == "optimal"
    assert sol.Z == a["objective"] and sol.iterations == a["iterations"]
    np.testing.assert_array_equal(sol.x[:lp["n"]], a["x"][:lp["n"]])


@pytest.mark.parametrize("text", [FREE1, FREE2, FREE3])
@pytest.mark.parametrize("dense", [0, 4096])
def test_free_columns_gpu_vs_oracle_and_highs(tmp_path, text, dense):
    p = S.Problem.readMps(write(tmp_path, text))
    h = highs_general(p)
    r = po.solve_typed(typed(p))
    s = S.CudaDualSimplex(S.Problem.readMps(write(tmp_path, text)), dense_max_m=dense)
    s.initDualSimplex()
    s.presolve("minInfeas")
    sol = s.solve()
    assert s.status() == "optimal"
    assert abs(sol.Z - h.fun) <= 1e-9 * max(1.0, abs(h.fun))
    assert abs(sol.Z - r["objective"]) <= 1e-12 * max(1.0, abs(h.fun))
