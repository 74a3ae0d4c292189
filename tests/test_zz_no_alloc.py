"""The allocation-free ratio test (ds_kernel_ratio_test_noalloc).

It serves callers that cannot call cudaMalloc (a framework that owns device
memory through its own pool, latency-critical loops where an allocation would
stall the device).  Its scratch is a fixed array inside the library, shared by
every call, so this checks two calls in a row against the allocating entry
point ds_kernel_ratio_test on the same vectors (bit-exact, the tolerance the
other ratio-test parity tests use), a call at exactly the size limit on a
caller's stream, that a call leaves the device's free memory unchanged, and
that an oversize input is rejected.
This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from parallel_ds_b200._lib import lib, ptr

pytestmark = pytest.mark.gpu


def case(seed, n, m):
    rng = np.random.default_rng(seed)
    N = n + m
    typ = rng.choice([0, 1, 2, 3, 4], size=N, p=[0.1, 0.05, 0.25, 0.2, 0.4]).astype(np.int32)
    lb = np.where(rng.random(N) < 0.5, 0.0, rng.standard_normal(N))
    ub = lb + rng.random(N) * 3
    ub[typ == 4] = 1e300
    lb[typ == 3] = -1e300
    x = np.where(rng.random(N) < 0.5, lb, ub)
    x = np.where(np.abs(x) > 1e100, 0.0, x)
    nonbasis = rng.permutation(N)[:n].astype(np.int32)
    alpha = rng.standard_normal(n) * (rng.random(n) < 0.6)
    d = np.abs(rng.standard_normal(N))
    d[rng.random(N) < 0.3] = 0.0
    delta = float(rng.standard_normal() * 3)
    return nonbasis, alpha, delta, int(delta < 0), x, d, lb, ub, typ


def with_alloc(nonbasis, alpha, delta, is_lower, x, d, lb, ub, typ):
    n, N = len(nonbasis), len(x)
    q, qi, nc = C.c_int(), C.c_int(), C.c_int()
    th, do = C.c_double(), C.c_double()
    IP, DP = C.c_int, C.c_double
    rc = lib().ds_kernel_ratio_test(n, N, ptr(nonbasis, IP), ptr(alpha, DP), delta, is_lower, ptr(x, DP),
                                    ptr(d, DP), ptr(lb, DP), ptr(ub, DP), ptr(typ, IP), C.byref(q),
                                    C.byref(qi), C.byref(th), C.byref(do), C.byref(nc))
    assert rc == 0
    return (q.value, qi.value, th.value, do.value, nc.value)


def on_device(nonbasis, alpha, delta, is_lower, x, d, lb, ub, typ):
    import torch
    dev = torch.device("cuda")
    t = {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in
         dict(nb=nonbasis, a=alpha, x=x, d=d, lb=lb, ub=ub, typ=typ.astype(np.uint8)).items()}
    torch.cuda.synchronize()
    return t, delta, is_lower


def call_noalloc(dev_args, stream=None):
    t, delta, is_lower = dev_args
    q, qi, nc = C.c_int(), C.c_int(), C.c_int()
    th, do = C.c_double(), C.c_double()
    rc = lib().ds_kernel_ratio_test_noalloc(t["nb"].numel(), t["x"].numel(), t["nb"].data_ptr(), t["a"].data_ptr(),
                                            delta, is_lower, t["x"].data_ptr(), t["d"].data_ptr(),
                                            t["lb"].data_ptr(), t["ub"].data_ptr(), t["typ"].data_ptr(),
                                            C.byref(q), C.byref(qi), C.byref(th), C.byref(do), C.byref(nc),
                                            stream)
    return rc, (q.value, qi.value, th.value, do.value, nc.value)


def without_alloc(*args):
    return call_noalloc(on_device(*args))


def test_noalloc_matches_allocating_entry_point_twice():
    # two calls in a row on the shared scratch: a large case, then a smaller one
    for seed, n, m in ((1, 40000, 20000), (2, 3000, 1500)):
        args = case(seed, n, m)
        rc, got = without_alloc(*args)
        assert rc == 0
        assert got == with_alloc(*args)


def test_noalloc_at_the_limit_on_a_caller_stream_allocates_nothing():
    import torch
    args = case(4, 65536, 4000)          # exactly DS_NOALLOC_MAX_SLOTS nonbasic slots
    dev_args = on_device(*args)
    want = with_alloc(*args)
    stream = torch.cuda.Stream()
    rc, got = call_noalloc(dev_args, C.c_void_p(stream.cuda_stream))   # warm: kernels loaded, address set up
    assert rc == 0 and got == want
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    rc, got = call_noalloc(dev_args, C.c_void_p(stream.cuda_stream))
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert rc == 0 and got == want
    assert free1 == free0


def test_noalloc_rejects_oversize():
    args = case(3, 70000, 10)
    rc, _ = without_alloc(*args)
    assert rc == -7   # DS_ERR_CAPACITY
