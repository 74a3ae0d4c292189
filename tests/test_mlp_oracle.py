"""Pins the network oracle (oracle/mlp_ref.py) on the CPU: its gradient
against central finite differences of its own FP64 loss, and its bfloat16
rounding against torch's conversion."""
import numpy as np

from oracle import mlp_ref as R


def _params(seed):
    r = np.random.default_rng(seed)
    p = np.zeros(R.NPARAMS)
    p[R.OFF_W1:R.OFF_B1] = r.normal(0, np.sqrt(2 / R.NF), R.H * R.NF)
    p[R.OFF_B1:R.OFF_W2] = r.normal(0, 0.1, R.H)
    p[R.OFF_W2:R.OFF_B2] = r.normal(0, np.sqrt(2 / R.H), R.H * R.H)
    p[R.OFF_B2:R.OFF_W3] = r.normal(0, 0.1, R.H)
    p[R.OFF_W3:R.OFF_B3] = r.normal(0, np.sqrt(1 / R.H), R.H)
    return p


def test_gradient_matches_finite_differences():
    r = np.random.default_rng(0)
    p = _params(1)
    X = r.normal(size=(50, R.NF))
    y = (r.random(50) < 0.5).astype(float)
    _, g = R.loss_and_grad(p, X, y)
    eps = 1e-6
    for k in list(r.choice(R.NPARAMS, 80, replace=False)) + [R.OFF_B3]:
        q = p.copy(); q[k] += eps
        lp = R.loss(R.forward(q, X, False)[0], y)
        q[k] -= 2 * eps
        lm = R.loss(R.forward(q, X, False)[0], y)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[k]) <= 1e-4 * (abs(fd) + abs(g[k])) + 1e-9, (k, fd, g[k])


def test_bf16_rounding_matches_torch():
    import torch
    r = np.random.default_rng(2)
    a = (r.normal(size=4000) * 10.0 ** r.integers(-6, 6, 4000)).astype(np.float32)
    a[:4] = [0.0, -0.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8]     # exact ties round to even
    ref = torch.tensor(a).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(R.bf16(a), ref)


def test_pdhg_restatement_approaches_the_optimum():
    """The PDHG oracle's estimate on a small generated LP comes close to the
    HiGHS optimum and identifies most of the optimal basis."""
    from conftest import highs
    from oracle import pdhg_ref as P
    from parallel_ds_b200 import lp as L
    lp = L.plain_small(seed=3)
    t = L.typed(lp)
    r = highs(lp)
    x, y = P.pdhg(t, 4000)
    assert abs(lp["c"] @ x - r.fun) <= 1e-2 * abs(r.fun)
    A = L.to_scipy(lp)
    slack = lp["b"] - A @ r.x
    basic = np.concatenate([r.x > 1e-9, slack > 1e-9])
    pred = np.concatenate([x > 1e-3, y <= 1e-3])
    assert np.mean(pred == basic) > 0.95
    gap, dual = P.evidence(t, x, y)
    assert np.all(np.isfinite(gap)) and np.all(dual >= 0)
