"""TEST INFRASTRUCTURE ONLY: a numpy restatement of the seeded LP generator.

It produces, bit for bit, the LPs that the product library's ds_gen_lp
(parallel_ds_b200/csrc/lp_gen.cpp) produces: min c^T x, A x <= b, x >= 0 with
N(0,1) entries, x0 ~ U[0,1]^n, b = A x0 + U[0.1,1]^m, c ~ U[0,1]^n, drawn from
a counter-based stream (the SplitMix64 finaliser over (seed, stream, index)).
bench.py's reference arm builds its inputs with it, so that the timed CPU
path loads nothing but the oracle; tests/test_lpgen.py pins it against the
library's generator.

Normal deviates use Box-Muller through Python's math module, which calls the
same C library log/cos/sqrt as the C++ generator, so the values are identical.
"""
import math

import numpy as np

M64 = (1 << 64) - 1
GOLD = 0x9E3779B97F4A7C15
S_STRUCT, S_VAL, S_X0, S_B, S_C, S_DIM = 1, 2, 3, 4, 5, 6
INF = 1e300
LOWER, UPPER = 4, 3

_U = np.uint64


def _mix_arr(z):
    z = (z ^ (z >> _U(30))) * _U(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> _U(27))) * _U(0x94D049BB133111EB)
    return z ^ (z >> _U(31))


def _mix(z):
    z &= M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def stream_key(seed, stream):
    return _mix(seed * GOLD + stream * 0xD1B54A32D192ED03 + 1)


def draws(key, idx):
    """draw(key, i) for an array of indices (uint64 arithmetic wraps)."""
    with np.errstate(over="ignore"):
        i = np.asarray(idx, dtype=np.uint64)
        return _mix_arr(_U(key) + (i + _U(1)) * _U(GOLD))


def draw(key, i):
    return _mix(key + (i + 1) * GOLD)


def u01(h):
    return float(h >> 11) * 2.0 ** -53


def normal(key, i):
    u1 = (float(draw(key, 2 * i) >> 11) + 1.0) * 2.0 ** -53
    u2 = u01(draw(key, 2 * i + 1))
    return math.sqrt(-2.0 * math.log(u1)) * math.cos(6.283185307179586476925 * u2)


def threshold(p):
    if p >= 1.0:
        return M64
    if p <= 0.0:
        return 0
    return int(p * 2.0 ** 64)


def _density_rows(seed, n, r0, r1, c0, c1, p, cols, vals):
    ks, kv = stream_key(seed, S_STRUCT), stream_key(seed, S_VAL)
    thr = _U(threshold(p))
    j = np.arange(c0, c1, dtype=np.uint64)
    for i in range(r0, r1):
        e = _U(i) * _U(n) + j
        hit = j[draws(ks, e) < thr] if thr < _U(M64) else j
        for jj in hit.tolist():
            cols[i].append(int(jj))
            vals[i].append(normal(kv, i * n + int(jj)))


def generate(kind=0, m=200, n=400, density=0.05, per_col=0, seed=0, blocks=0, block_m=0, block_n=0,
             link_rows=0, block_density=0.0, link_density=0.0):
    """dict(m, n, row_ptr, col_idx, val, b, c, seed) like parallel_ds_b200.lp.generate."""
    cols = [[] for _ in range(m)]
    vals = [[] for _ in range(m)]
    if kind == 0:
        _density_rows(seed, n, 0, m, 0, n, density, cols, vals)
    elif kind == 1:
        ks, kv = stream_key(seed, S_STRUCT), stream_key(seed, S_VAL)
        for jj in range(n):
            got, t = [], 0
            while len(got) < per_col:
                cand = draw(ks, jj * 4096 + t) % m
                t += 1
                if cand not in got:
                    got.append(cand)
            for s, i in enumerate(got):
                cols[i].append(jj)
                vals[i].append(normal(kv, jj * per_col + s))
    elif kind == 2:
        for blk in range(blocks):
            _density_rows(seed, n, blk * block_m, (blk + 1) * block_m, blk * block_n, (blk + 1) * block_n,
                          block_density, cols, vals)
        _density_rows(seed, n, blocks * block_m, m, 0, n, link_density, cols, vals)
    else:
        raise ValueError("unknown generator kind")
    row_ptr = np.zeros(m + 1, np.int32)
    ci, va = [], []
    for i in range(m):
        order = sorted(range(len(cols[i])), key=lambda t: cols[i][t])
        ci += [cols[i][t] for t in order]
        va += [vals[i][t] for t in order]
        row_ptr[i + 1] = len(ci)
    col_idx = np.asarray(ci, np.int32)
    val = np.asarray(va, np.float64)
    kx, kb, kc = stream_key(seed, S_X0), stream_key(seed, S_B), stream_key(seed, S_C)
    x0 = [u01(draw(kx, j)) for j in range(n)]
    b = np.zeros(m)
    for i in range(m):
        s = 0.0
        for e in range(row_ptr[i], row_ptr[i + 1]):
            s += va[e] * x0[ci[e]]
        b[i] = s + (0.1 + 0.9 * u01(draw(kb, i)))
    c = np.asarray([u01(draw(kc, j)) for j in range(n)])
    return dict(m=m, n=n, row_ptr=row_ptr, col_idx=col_idx, val=val, b=b, c=c, seed=seed)


def learned(seed=0):
    return generate(0, 2000, 4000, density=0.01, seed=seed)


def plain_small(seed=0):
    return generate(0, 200, 400, density=0.05, seed=seed)


def typed(lp):
    """The reference's typed form of A x <= b, x >= 0 (as parallel_ds_b200.lp.typed)."""
    m, n = lp["m"], lp["n"]
    return dict(m=m, n=n, row_ptr=lp["row_ptr"], col_idx=lp["col_idx"], val=lp["val"], c=lp["c"],
                col_type=np.full(n, LOWER, np.int32), col_lb=np.zeros(n), col_ub=np.full(n, INF),
                row_type=np.full(m, UPPER, np.int32), row_lb=np.full(m, -INF), row_ub=np.asarray(lp["b"], float))


def batch_m(seed, i, m_lo, m_hi):
    """Row count of instance i of a batch (ds_gen_batch_m)."""
    if m_hi < m_lo:
        return m_lo
    return m_lo + draw(stream_key(seed + i, S_DIM), 0) % (m_hi - m_lo + 1)


def batched_instance(seed, i, m_lo=32, m_hi=512, density=0.10):
    m = batch_m(seed, i, m_lo, m_hi)
    return generate(0, m, 2 * m, density=density, seed=seed + i)
