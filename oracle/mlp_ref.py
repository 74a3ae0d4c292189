"""TEST INFRASTRUCTURE ONLY: FP64 numpy restatement of the leaving-row network.

Checks the tensor-core forward / backward kernels of csrc/mlp.cu.  The network
has no counterpart in the reference; this file states the mathematics the
kernels implement:

    h1 = relu(X W1^T + b1),  h2 = relu(h1 W2^T + b2),  z = h2 . w3 + b3
    loss = mean over rows of  max(z, 0) - z y + log(1 + exp(-|z|))

With ``rounding=True`` the operands of every tensor-core product are rounded
to bfloat16 (round to nearest even) exactly where the kernels round them:
X, W1 and W2, h1 before the second layer, and in the backward pass dH2, H1,
dH1 and X before the three gradient products.  Biases, w3, the activations
themselves and every accumulation stay in FP64 here (FP32 on the GPU).
"""
import numpy as np

NF = 12
H = 64
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * NF
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
NPARAMS = OFF_B3 + 1


def bf16(a):
    """Round to bfloat16 (nearest, ties to even) through float32, returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def _r(a, rounding):
    return bf16(a) if rounding else np.asarray(a, dtype=np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(H, NF), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3], p[OFF_B3])


def layer1(p, X, rounding=True):
    W1, b1, _, _, _, _ = unpack(p)
    return np.maximum(_r(X, rounding) @ _r(W1, rounding).T + b1, 0.0)


def layer2(p, H1, rounding=True):
    _, _, W2, b2, _, _ = unpack(p)
    return np.maximum(_r(H1, rounding) @ _r(W2, rounding).T + b2, 0.0)


def head(p, H2):
    _, _, _, _, w3, b3 = unpack(p)
    return H2 @ w3 + b3


def forward(p, X, rounding=True):
    H1 = layer1(p, X, rounding)
    H2 = layer2(p, H1, rounding)
    return head(p, H2), H1, H2


def loss(z, y):
    z = np.asarray(z, np.float64)
    return float(np.mean(np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z)))))


def backward(p, X, y, H1, H2, z, rounding=True):
    """Gradient of the mean loss (flat, parameter order) given the forward
    activations (from this file or from the GPU)."""
    _, _, W2, _, w3, _ = unpack(p)
    M = X.shape[0]
    z = np.asarray(z, np.float64)
    g3 = (1.0 / (1.0 + np.exp(-z)) - y) / M                   # d loss / d z
    dH2 = np.where(np.asarray(H2) > 0, g3[:, None] * w3[None, :], 0.0)
    dH1 = _r(dH2, rounding) @ _r(W2, rounding)
    dH1 = np.where(np.asarray(H1) > 0, dH1, 0.0)
    g = np.zeros(NPARAMS)
    g[OFF_W2:OFF_B2] = (_r(dH2, rounding).T @ _r(H1, rounding)).ravel()
    g[OFF_W1:OFF_B1] = (_r(dH1, rounding).T @ _r(X, rounding)).ravel()
    g[OFF_B2:OFF_W3] = dH2.sum(0)
    g[OFF_B1:OFF_W2] = dH1.sum(0)
    g[OFF_W3:OFF_B3] = (g3[:, None] * np.asarray(H2, np.float64)).sum(0)
    g[OFF_B3] = g3.sum()
    return g


def loss_and_grad(p, X, y, rounding=False):
    z, H1, H2 = forward(p, X, rounding)
    return loss(z, y), backward(p, X, y, H1, H2, z, rounding)
