"""Host stage of the eta-file mode's sparse LU: the singleton triangularisation
(ds_sparse_triangularise, no GPU needed).  Checked by its defining property:
with rows and columns in the returned order the pattern is block upper
triangular, [U1 X Y; 0 M Z; 0 0 U3], with the singleton pivots on the diagonal;
and by the known kernels of small patterns."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from parallel_ds_b200._lib import lib, ptr

DS_ERR_NUMERIC = -5


def triangularise(A):
    A = sp.csc_matrix(A)
    A.sort_indices()
    k = A.shape[0]
    ro, co = np.zeros(k, np.int32), np.zeros(k, np.int32)
    c1, km = C.c_int(), C.c_int()
    rc = lib().ds_sparse_triangularise(k, ptr(A.indptr.astype(np.int32), C.c_int),
                                       ptr(A.indices.astype(np.int32), C.c_int), ptr(ro, C.c_int), ptr(co, C.c_int),
                                       C.byref(c1), C.byref(km))
    return rc, ro, co, c1.value, km.value


def check_block_triangular(A, ro, co, c1, km):
    k = A.shape[0]
    assert sorted(ro) == list(range(k)) and sorted(co) == list(range(k))
    pr, pc = np.empty(k, int), np.empty(k, int)
    pr[ro] = np.arange(k)
    pc[co] = np.arange(k)
    B = sp.coo_matrix(A)
    r, c = pr[B.row], pc[B.col]
    kern = (r >= c1) & (r < c1 + km)
    assert np.all(c[~kern] >= r[~kern])            # U1 and U3 rows: upper triangular
    assert np.all(c[kern] >= c1)                   # kernel rows: nothing in U1's columns
    diag = set(zip(r.tolist(), c.tolist()))
    for p in list(range(c1)) + list(range(c1 + km, k)):
        assert (p, p) in diag                      # singleton pivots sit on the diagonal


@pytest.mark.parametrize("seed", range(6))
def test_random_permuted_patterns(seed):
    """Random nonsingular patterns (a diagonal plus random entries, rows and
    columns shuffled) at the densities of the large workload's bumps."""
    rng = np.random.default_rng(seed)
    k = int(rng.integers(50, 3000))
    extra = rng.uniform(0.2, 2.5)
    nz = int(extra * k)
    rows = np.concatenate([np.arange(k), rng.integers(0, k, nz)])
    cols = np.concatenate([np.arange(k), rng.integers(0, k, nz)])
    A = sp.csc_matrix((np.ones(len(rows)), (rows, cols)), shape=(k, k))
    A = A[rng.permutation(k)][:, rng.permutation(k)]
    rc, ro, co, c1, km = triangularise(A)
    assert rc == 0
    check_block_triangular(A, ro, co, c1, km)


def test_triangular_pattern_has_no_kernel():
    A = sp.triu(sp.random(200, 200, density=0.03, random_state=1) + sp.identity(200)).tocsc()
    rc, ro, co, c1, km = triangularise(A)
    assert rc == 0 and km == 0
    check_block_triangular(A, ro, co, c1, km)


def test_dense_block_is_the_kernel():
    """A dense 5 x 5 block behind a triangular part: the kernel is the block."""
    k = 12
    A = np.zeros((k, k))
    A[:5, :5] = 1.0
    for i in range(5, k):
        A[i, i] = 1.0
        A[i - 1, i] = 1.0
    rc, ro, co, c1, km = triangularise(A)
    assert rc == 0 and km == 5
    check_block_triangular(sp.csc_matrix(A), ro, co, c1, km)


@pytest.mark.parametrize("case", ["empty_column", "shared_singleton_row"])
def test_structurally_singular(case):
    A = np.eye(6)
    if case == "empty_column":
        A[:, 2] = 0.0
        A[2, 3] = 1.0
    else:                                          # columns 0 and 1 both only in row 0
        A[:, 1] = 0.0
        A[0, 1] = 1.0
        A[1, 4] = 1.0
    rc, *_ = triangularise(A)
    assert rc == DS_ERR_NUMERIC


def test_malformed_pattern_rejected():
    k = 3
    ro, co = np.zeros(k, np.int32), np.zeros(k, np.int32)
    c1, km = C.c_int(), C.c_int()
    for ptr_, idx in (([0, 2, 1, 3], [0, 1, 2]), ([1, 2, 3, 4], [0, 1, 2, 0]), ([0, 1, 2, 3], [0, 5, 2])):
        p_ = np.asarray(ptr_, np.int32)
        i_ = np.asarray(idx, np.int32)
        rc = lib().ds_sparse_triangularise(k, ptr(p_, C.c_int), ptr(i_, C.c_int), ptr(ro, C.c_int),
                                           ptr(co, C.c_int), C.byref(c1), C.byref(km))
        assert rc == -1                            # DS_ERR_ARG
