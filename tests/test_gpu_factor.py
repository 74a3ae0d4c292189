"""GPU refactorisation + FTRAN/BTRAN against dense numpy solves.

Bases come from the oracle's own trajectory (so they are the nonsingular bases
the dual simplex visits), at several iteration counts so that the structural
block k spans small to large sizes.  Tolerance: 1e-10 relative to the solution
scale (the bases have condition numbers around 1e3-1e4)."""
import ctypes as C

import numpy as np
import pytest

from oracle import pyoracle as po
from parallel_ds_b200 import lp as L
from parallel_ds_b200._lib import FACTOR_DENSE, FACTOR_SPARSE, DsOptions, lib, ptr

pytestmark = pytest.mark.gpu


def dense_basis(lp, basis):
    m, n = lp["m"], lp["n"]
    A = L.to_scipy(lp).toarray()
    B = np.zeros((m, m))
    for i, v in enumerate(basis):
        if v < n:
            B[:, i] = A[:, v]
        else:
            B[v - n, i] = 1.0
    return B


def solver_options(mode):
    """"dense": the explicit B^-1 of dense mode (Gauss-Jordan of the bump);
    "sparse": eta-file mode with the sparse LU of the bump;
    "eta_gj": eta-file mode with the Gauss-Jordan inverse of the bump."""
    o = DsOptions()
    lib().ds_default_options(C.byref(o))
    if mode != "dense":
        o.dense_max_m = 0
        o.factor_mode = FACTOR_DENSE if mode == "eta_gj" else FACTOR_SPARSE
    return o


MODES = ["dense", "sparse", "eta_gj"]


def gpu_solve(lp, basis, rhs, transpose, mode="dense"):
    t = L.typed(lp)
    L_ = lib()
    h = C.c_void_p()
    o = solver_options(mode)
    assert L_.ds_create(C.byref(o), C.byref(h)) == 0
    try:
        rc = L_.ds_load_typed(h, t["m"], t["n"], ptr(t["row_ptr"], C.c_int), ptr(t["col_idx"], C.c_int),
                              ptr(t["val"], C.c_double), ptr(t["c"], C.c_double), ptr(t["col_type"], C.c_int),
                              ptr(t["col_lb"], C.c_double), ptr(t["col_ub"], C.c_double),
                              ptr(t["row_type"], C.c_int), ptr(t["row_lb"], C.c_double),
                              ptr(t["row_ub"], C.c_double))
        assert rc == 0
        b = np.ascontiguousarray(basis, np.int32)
        r = np.ascontiguousarray(rhs.T if rhs.ndim == 2 else rhs[None, :], np.float64)
        out = np.zeros_like(r)
        rc = L_.ds_basis_solve(h, ptr(b, C.c_int), ptr(r, C.c_double), ptr(out, C.c_double), r.shape[0],
                               int(transpose))
        assert rc == 0, L_.ds_last_error(h)
    finally:
        L_.ds_destroy(h)
    return out.T if rhs.ndim == 2 else out[0]


@pytest.fixture(scope="module")
def learned_bases():
    lp = L.learned(0)
    t = L.typed(lp)
    out = []
    for it in (1, 150, 300, 376, 700, 1500):
        r = po.solve_typed(t, max_iterations=it)
        out.append((it, r["basis"]))
    return lp, out


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("transpose", [0, 1])
def test_basis_solve_dense_rhs(learned_bases, transpose, mode):
    lp, bases = learned_bases
    rng = np.random.default_rng(1)
    for it, basis in bases:
        B = dense_basis(lp, basis)
        rhs = rng.standard_normal((lp["m"], 3))
        ref = np.linalg.solve(B.T if transpose else B, rhs)
        got = gpu_solve(lp, basis, rhs, transpose, mode)
        k = int((basis < lp["n"]).sum())
        err = np.abs(got - ref).max() / max(1.0, np.abs(ref).max())
        assert err <= 1e-10, (it, k, err)


@pytest.mark.parametrize("mode", MODES)
def test_basis_solve_sparse_and_unit_rhs(learned_bases, mode):
    lp, bases = learned_bases
    A = L.to_scipy(lp).tocsc()
    for it, basis in bases[1:]:
        B = dense_basis(lp, basis)
        cols = [A[:, j].toarray().ravel() for j in (0, 17, 3999)] + [np.eye(lp["m"])[5]]
        rhs = np.stack(cols, axis=1)
        ref = np.linalg.solve(B, rhs)
        got = gpu_solve(lp, basis, rhs, 0, mode)
        err = np.abs(got - ref).max() / max(1.0, np.abs(ref).max())
        assert err <= 1e-10, (it, err)


@pytest.mark.parametrize("mode", ["dense", "sparse"])
@pytest.mark.parametrize("nr", [1, 2, 3, 4, 5])
def test_basis_solve_rhs_counts(learned_bases, nr, mode):
    lp, bases = learned_bases
    it, basis = bases[3]
    B = dense_basis(lp, basis)
    rhs = np.random.default_rng(nr).standard_normal((lp["m"], nr))
    ref = np.linalg.solve(B, rhs)
    got = gpu_solve(lp, basis, rhs, 0, mode)
    assert np.abs(got - ref).max() <= 1e-10 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("k", [1601, 2400])
def test_basis_solve_bump_above_shared_memory_panel(k, mode):
    """A structural bump larger than the shared-memory panel limit (1600 rows),
    so the Gauss-Jordan panels run from global memory: random structural columns
    of a sparse 1%-dense LP plus slacks for the other rows, checked against a
    dense solve."""
    m = k + 600
    lp = L.generate(m=m, n=2 * m, density=0.01, seed=k)
    r = np.random.default_rng(k)
    cols = np.sort(r.choice(lp["n"], size=k, replace=False))
    slack_rows = np.sort(r.choice(m, size=m - k, replace=False))
    basis = np.concatenate([cols, lp["n"] + slack_rows]).astype(np.int32)
    r.shuffle(basis)
    B = dense_basis(lp, basis)
    assert np.linalg.matrix_rank(B) == m            # a nonsingular basis
    rhs = r.normal(size=m)
    for transpose in (0, 1):
        x = gpu_solve(lp, basis, rhs, transpose, mode)
        ref = np.linalg.solve(B.T if transpose else B, rhs)
        assert np.max(np.abs(x - ref)) <= 1e-9 * (1 + np.max(np.abs(ref))), transpose


def sparse_basis_matrix(lp, basis):
    import scipy.sparse as sp
    m, n = lp["m"], lp["n"]
    A = L.to_scipy(lp).tocsc()
    cols = []
    for v in basis:
        cols.append(A[:, v] if v < n else sp.csc_matrix(([1.0], ([v - n], [0])), shape=(m, 1)))
    return sp.hstack(cols).tocsc()


@pytest.fixture(scope="module")
def per_col_bases():
    """Bases the sparse-LU solver visits on a 10,000 x 20,000 LP with 8
    nonzeros per column (the large eta-file workload's generator at a fifth of
    its size): structural bumps of several thousand columns."""
    from parallel_ds_b200 import solver as S
    lp = L.generate(L._lib.GEN_PER_COL, 10000, 20000, per_col=8, seed=5)
    out = []
    for it in (1500, 4000, 7000):
        r = S.solve_lp(lp, max_iterations=it, dense_max_m=0)
        out.append((it, r["basis"], r["stats"]))
    return lp, out


@pytest.mark.parametrize("transpose", [0, 1])
def test_sparse_lu_large_bumps(per_col_bases, transpose):
    """ds_basis_solve through the sparse LU on visited bases with bumps of
    thousands of columns.  These bases are ill-conditioned (forward errors of
    scipy's own sparse LU reach 1e-9), so the bar is the backward error
    |B x - b| / (|B| |x| + |b|) <= 1e-13 (infinity norms), the same bar scipy's
    splu meets on them."""
    from scipy.sparse.linalg import splu
    lp, bases = per_col_bases
    rng = np.random.default_rng(7)
    ks = []
    for it, basis, _ in bases:
        B = sparse_basis_matrix(lp, basis)
        M = B.T.tocsc() if transpose else B
        nb = abs(M).sum(axis=1).max()
        rhs = rng.standard_normal((lp["m"], 2))
        got = gpu_solve(lp, basis, rhs, transpose, "sparse")
        lu = splu(M)
        for q in range(2):
            for x in (got[:, q], lu.solve(rhs[:, q])):
                berr = np.abs(M @ x - rhs[:, q]).max() / (nb * np.abs(x).max() + np.abs(rhs[:, q]).max())
                assert berr <= 1e-13, (it, berr)
        ks.append(int((basis < lp["n"]).sum()))
    assert max(ks) >= 3000, ks
