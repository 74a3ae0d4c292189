"""MPS reader (ds_mps_read, Problem.readMps) on the CPU.

The reference reads MPS through Clp (ClpModel::readMps / CoinUtils' CoinMpsIO,
absent here), then derives bound types in Problem::readMps
(problem.tpp:332-409).  These tests pin the reader to the MPS format's rules
on hand-written files whose arrays are worked out by hand, to exact round
trips of generated LPs, and to HiGHS optima of the parsed LPs solved by the
CPU oracle."""
import numpy as np
import pytest
from scipy.optimize import linprog

from oracle import pyoracle as po
from parallel_ds_b200 import lp as L
from parallel_ds_b200 import solver as S
from parallel_ds_b200._lib import DsError

INF = 1e300

SAMPLE = """NAME          TESTLP
* a comment line
ROWS
 N  COST
 L  LIM1
 G  LIM2
 E  MYEQN
 N  SPARE
COLUMNS
    MARKER                 'MARKER'                 'INTORG'
    X1        COST         1.0   LIM1         1.0
    X1        LIM2         1.0   SPARE        9.0
    MARKER                 'MARKER'                 'INTEND'
    X2        COST         2.0   LIM1         1.0
    X2        MYEQN       -1.0
    X3        COST        -1.0   MYEQN        1.0
    X4        LIM2        -2.0
RHS
    RHS       COST        -3.5
    RHS       LIM1         4.0   LIM2         1.0
    RHS       MYEQN        7.0
    RHS2      LIM1       100.0
RANGES
    RNG       LIM1         2.5   MYEQN       -2.0
BOUNDS
 UP BND       X1           4.0
 LO BND       X2          -1.0
 UP BND       X2           1.0
 FR BND       X3
 UP BND       X4          -2.0
 UP BND2      X1           9.0
ENDATA
"""


def write(tmp_path, text, name="t.mps"):
    f = tmp_path / name
    f.write_text(text)
    return f


def test_sample_by_hand(tmp_path):
    p = S.Problem.readMps(write(tmp_path, SAMPLE))
    # rows LIM1 [4-2.5, 4], LIM2 [1, inf), MYEQN (E, range -2) [5, 7]; SPARE (N) dropped
    np.testing.assert_array_equal(p.A.row_ptr, [0, 2, 4, 6])
    np.testing.assert_array_equal(p.A.col_id, [0, 1, 0, 3, 1, 2])
    np.testing.assert_array_equal(p.A.val, [1.0, 1.0, 1.0, -2.0, -1.0, 1.0])
    np.testing.assert_array_equal(p.costs, [1.0, 2.0, -1.0, 0.0])
    np.testing.assert_array_equal(p.lower_range, [1.5, 1.0, 5.0])
    np.testing.assert_array_equal(p.upper_range, [4.0, INF, 7.0])
    # X1 [0,4] (second BOUNDS set ignored), X2 [-1,1], X3 free, X4 UP<0 on a default lower -> (-inf, -2]
    np.testing.assert_array_equal(p.lower_bound, [0.0, -1.0, -INF, -INF])
    np.testing.assert_array_equal(p.upper_bound, [4.0, 1.0, INF, -2.0])
    B = S.BoundaryType
    assert list(p.bound_type) == [B.Boxed, B.Boxed, B.Free, B.Upper]
    assert list(p.range_type) == [B.Boxed, B.Lower, B.Boxed]
    assert p._offset == -3.5


def test_free_format_and_bound_kinds(tmp_path):
    text = """NAME free
ROWS
N obj
G r1
L r2
COLUMNS
a obj 1 r1 1
b obj 1 r1 1
b r2 1
c obj 3 r2 2
d obj 1 r1 1
RHS
r1 2 r2 1e30
BOUNDS
BV BND a
MI BND b
FX BND c 0.25
PL BND d
LO BND d 1.5
ENDATA
"""
    p = S.Problem.readMps(write(tmp_path, text))
    assert (p.A.m, p.A.n) == (2, 4)
    np.testing.assert_array_equal(p.lower_bound, [0.0, -INF, 0.25, 1.5])
    np.testing.assert_array_equal(p.upper_bound, [1.0, INF, 0.25, INF])
    np.testing.assert_array_equal(p.lower_range, [2.0, -INF])
    np.testing.assert_array_equal(p.upper_range, [INF, INF])   # rhs 1e30 is infinite
    B = S.BoundaryType
    assert list(p.bound_type) == [B.Boxed, B.Free, B.Fixed, B.Lower]   # MI keeps the default +inf upper
    assert list(p.range_type) == [B.Lower, B.Free]


@pytest.mark.parametrize("text,msg", [
    ("NAME x\nROWS\n N obj\nOBJSENSE\n    MAX\nENDATA\n", "OBJSENSE MAX"),
    ("NAME x\nROWS\n N obj\n L r\nCOLUMNS\n    x obj 1 q 1\nENDATA\n", "unknown row q"),
    ("NAME x\nROWS\n N obj\n L r\nCOLUMNS\n    x obj 1 r 1\n", "without ENDATA"),
    ("NAME x\nROWS\n N obj\n L r\nCOLUMNS\n    x r 1\nBOUNDS\n SC BND x 3\nENDATA\n", "unsupported bound type SC"),
    ("NAME x\nROWS\n N obj\n L r\nCOLUMNS\n    x r 1 r 2\nENDATA\n", "duplicate entry"),
    ("NAME x\nROWS\n L r\nCOLUMNS\n    x r 1\nENDATA\n", "no objective"),
])
def test_errors(tmp_path, text, msg):
    with pytest.raises(DsError, match=msg):
        S.Problem.readMps(write(tmp_path, text))


def test_missing_file(tmp_path):
    with pytest.raises(DsError, match="cannot open"):
        S.Problem.readMps(tmp_path / "absent.mps")


def to_mps(lp, name="GEN"):
    """Fixed-layout MPS of a generated LP (min c^T x, A x <= b, x >= 0), values in repr form."""
    m, n = lp["m"], lp["n"]
    rp, ci, va = lp["row_ptr"], lp["col_idx"], lp["val"]
    cols = [[] for _ in range(n)]
    for i in range(m):
        for e in range(rp[i], rp[i + 1]):
            cols[ci[e]].append((i, va[e]))
    out = [f"NAME          {name}", "ROWS", " N  OBJ"] + [f" L  R{i}" for i in range(m)] + ["COLUMNS"]
    for j in range(n):
        out.append(f"    C{j}  OBJ  {float(lp['c'][j])!r}")
        out += [f"    C{j}  R{i}  {float(v)!r}" for i, v in cols[j]]
    out += ["RHS"] + [f"    RHS  R{i}  {float(b)!r}" for i, b in enumerate(lp["b"])] + ["ENDATA"]
    return "\n".join(out) + "\n"


@pytest.mark.parametrize("seed", [0, 3])
def test_round_trip_of_generated_lp(tmp_path, seed):
    lp = L.plain_small(seed)
    p = S.Problem.readMps(write(tmp_path, to_mps(lp)))
    np.testing.assert_array_equal(p.A.row_ptr, lp["row_ptr"])
    np.testing.assert_array_equal(p.A.col_id, lp["col_idx"])
    np.testing.assert_array_equal(p.A.val, lp["val"])
    np.testing.assert_array_equal(p.costs, lp["c"])
    np.testing.assert_array_equal(p.upper_range, lp["b"])
    assert np.all(p.lower_range == -INF) and np.all(p.lower_bound == 0) and np.all(p.upper_bound == INF)


def typed(p):
    return dict(m=p.A.m, n=p.A.n, row_ptr=p.A.row_ptr, col_idx=p.A.col_id, val=p.A.val, c=p.costs,
                col_type=p.bound_type, col_lb=p.lower_bound, col_ub=p.upper_bound,
                row_type=p.range_type, row_lb=p.lower_range, row_ub=p.upper_range)


def highs_general(p):
    """HiGHS on row_lb <= A x <= row_ub, col_lb <= x <= col_ub."""
    from scipy.sparse import csr_matrix
    A = csr_matrix((p.A.val, p.A.col_id, p.A.row_ptr), shape=(p.A.m, p.A.n))
    up, lo = p.upper_range < 1e100, p.lower_range > -1e100
    from scipy.sparse import vstack
    A_ub = vstack([A[up], -A[lo]])
    b_ub = np.concatenate([p.upper_range[up], -p.lower_range[lo]])
    bnd = [(None if l < -1e100 else l, None if u > 1e100 else u) for l, u in zip(p.lower_bound, p.upper_bound)]
    return linprog(p.costs, A_ub=A_ub, b_ub=b_ub, bounds=bnd, method="highs-ds")


# The sample without its free column, and three-line LPs with free columns.
# Free structural columns go through the solver's crash (default mode): the
# reference's phase 1 alone (strict_reference) stops with a dual infeasible
# basis on them -- "primal infeasible" on the sample, 0 instead of -5 on FREE1.
SAMPLE_SOLVE = SAMPLE.replace(" FR BND       X3\n", "")
FREE1 = "NAME a\nROWS\n N obj\n L r1\nCOLUMNS\n    x obj -1 r1 1\nRHS\n    RHS r1 5\nBOUNDS\n FR B x\nENDATA\n"
FREE2 = ("NAME a\nROWS\n N obj\n L r1\n G r2\nCOLUMNS\n    x obj -1 r1 1\n    y obj 1 r1 1\n    y r2 1\n"
         "RHS\n    RHS r1 5 r2 1\nBOUNDS\n FR B x\nENDATA\n")
FREE3 = ("NAME a\nROWS\n N obj\n E r1\nCOLUMNS\n    x obj -1 r1 -1\n    y obj 2 r1 1\nRHS\n    RHS r1 3\n"
         "BOUNDS\n FR B x\n UP B y 10\nENDATA\n")


@pytest.mark.parametrize("text", [SAMPLE, FREE1, FREE2, FREE3])
def test_free_columns_oracle_vs_highs(tmp_path, text):
    p = S.Problem.readMps(write(tmp_path, text))
    h = highs_general(p)
    r = po.solve_typed(typed(p))
    assert h.status == 0 and r["status"] == "optimal"
    assert abs(r["objective"] - h.fun) <= 1e-9 * max(1.0, abs(h.fun))


def test_free_column_strict_reference_keeps_the_reference_phase1(tmp_path):
    r = po.solve_typed(typed(S.Problem.readMps(write(tmp_path, FREE1))), strict_reference=1)
    assert r["status"] == "optimal" and r["objective"] == 0.0   # HiGHS: -5


def test_parsed_sample_solves_to_highs_optimum(tmp_path):
    """The hand-written LP through the CPU oracle (the reference's algorithm) and
    HiGHS, with an (-inf, -2] column, ranged rows and an equality range."""
    p = S.Problem.readMps(write(tmp_path, SAMPLE_SOLVE))
    h = highs_general(p)
    r = po.solve_typed(typed(p))
    assert h.status == 0 and r["status"] == "optimal"
    assert abs(r["objective"] - h.fun) <= 1e-9 * max(1.0, abs(h.fun))
    assert abs(h.fun - (-5.5)) <= 1e-9   # X1 + X2 - 7 at X1 + X2 = 1.5
