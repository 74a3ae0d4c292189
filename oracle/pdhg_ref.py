"""TEST INFRASTRUCTURE ONLY: numpy restatement of the PDHG warm-start estimate.

Checks csrc/pdhg.cu.  No counterpart in the reference; this follows the
published method: primal-dual hybrid gradient (Chambolle & Pock 2011) for
min c^T x s.t. L <= A x <= U, lo <= x <= hi, with the diagonal steps of
Pock & Chambolle (2011, alpha = 1) and a restart to the running average every
R iterations.  Bounds come from the typed LP (ds_load_typed form) the way the
engine reads them: a bound exists only where the type has it, a FIXED
variable is pinned to its lower bound, and row activity bounds are the negated
slack bounds (the slack is s = -A x with bounds [-row_ub, -row_lb]).
"""
import numpy as np
import scipy.sparse as sp

FIXED, FREE, BOXED, UPPER, LOWER = 0, 1, 2, 3, 4
INF = np.inf


def _lower(t, lb):
    return np.where((t == FIXED) | (t == BOXED) | (t == LOWER), lb, -INF)


def _upper(t, lb, ub):
    return np.where(t == FIXED, lb, np.where((t == BOXED) | (t == UPPER), ub, INF))


# row type (DS_* of the row) -> slack type, as the engine maps them
_SLACK = {FIXED: FIXED, BOXED: BOXED, LOWER: UPPER, UPPER: LOWER, FREE: FREE}


def bounds(t):
    """(lo, hi, L, U) of a typed LP dict."""
    ct = np.asarray(t["col_type"])
    lo = _lower(ct, np.asarray(t["col_lb"], float))
    hi = _upper(ct, np.asarray(t["col_lb"], float), np.asarray(t["col_ub"], float))
    st = np.array([_SLACK.get(int(r), FREE) for r in t["row_type"]])
    slb = -np.asarray(t["row_ub"], float)
    sub = -np.asarray(t["row_lb"], float)
    return lo, hi, -_upper(st, slb, sub), -_lower(st, slb)


def pdhg(t, iters, R=500):
    """x, y after ceil(iters / R) restart periods (y: row duals, c + A^T y reduced costs)."""
    m, n = int(t["m"]), int(t["n"])
    A = sp.csr_matrix((t["val"], t["col_idx"], t["row_ptr"]), shape=(m, n))
    c = np.asarray(t["c"], float)
    lo, hi, L, U = bounds(t)
    cs = np.asarray(abs(A).sum(0)).ravel()
    rs = np.asarray(abs(A).sum(1)).ravel()
    tau = np.where(cs > 0, 1.0 / np.where(cs > 0, cs, 1.0), 1.0)
    sig = np.where(rs > 0, 1.0 / np.where(rs > 0, rs, 1.0), 1.0)
    AT = A.T.tocsr()
    x = np.clip(0.0, lo, hi) * np.ones(n)
    y = np.zeros(m)
    xsum = R * x
    ysum = np.zeros(m)
    periods = (iters + R - 1) // R
    for _ in range(periods):
        for k in range(R):
            if k == 0:
                x = xsum / R
                xsum = np.zeros(n)
            xn = np.clip(x - tau * (c + AT @ y), lo, hi)
            xbar = 2 * xn - x
            x = xn
            xsum += xn
            v = y + sig * (A @ xbar)
            y = v - sig * np.clip(v / sig, L, U)
            ysum += y
            if k == R - 1:
                y = ysum / R
                ysum = np.zeros(m)
    x = xsum / R
    return x, y


def evidence(t, x, y):
    """(gap, dual) per variable (structurals then slacks), as the scorer reads them."""
    m, n = int(t["m"]), int(t["n"])
    A = sp.csr_matrix((t["val"], t["col_idx"], t["row_ptr"]), shape=(m, n))
    lo, hi, L, U = bounds(t)
    act = A @ x
    gap = np.concatenate([np.minimum(x - lo, hi - x), np.minimum(act - L, U - act)])
    dual = np.concatenate([np.abs(np.asarray(t["c"], float) + A.T @ y), np.abs(y)])
    return np.minimum(gap, 1e30), dual
