"""FP64 numpy restatement of the learned relaxation-time network and its
training step: the checker of the CUDA training kernels (tau_train.cu) and of
the fused inference (lbm_common.cuh learned_tau).  Test infrastructure only.

There is no reference code for this part (the reference's relaxation-time
networks are the TorchScript boundary nets).  The network: x (6 standardised
features) -> h1 = tanh(W1 x + b1) (32) -> h2 = tanh(W2 h1 + b2) (32) ->
z = w3 . h2 + b3 -> softplus(z).  Parameters flat, row-major (out x in):
W1[32][6] b1[32] W2[32][32] b2[32] w3[32] b3.  Loss: mean squared error of
softplus(z) against the targets.  Parity is pinned by finite differences of
this restatement (tests/test_tau_mlp.py) and by the closed forms below.
"""
from __future__ import annotations

import numpy as np

NIN, NHID = 6, 32
W1, B1 = 0, 192
W2, B2 = 224, 1248
W3, B3 = 1280, 1312
NPARAM = 1313


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    return (w[W1:B1].reshape(NHID, NIN), w[B1:W2], w[W2:B2].reshape(NHID, NHID), w[B2:W3],
            w[W3:B3], w[B3])


def softplus(z):
    return np.maximum(z, 0.0) + np.log1p(np.exp(-np.abs(z)))


def forward(w, x):
    """softplus(MLP(x)) for x[n][6]."""
    a1, c1, a2, c2, v3, c3 = unpack(w)
    h1 = np.tanh(x @ a1.T + c1)
    h2 = np.tanh(h1 @ a2.T + c2)
    return softplus(h2 @ v3 + c3)


def loss_and_grad(w, x, y):
    """Mean squared error of softplus(MLP(x)) against y and its gradient."""
    a1, c1, a2, c2, v3, c3 = unpack(w)
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    n = x.shape[0]
    h1 = np.tanh(x @ a1.T + c1)
    h2 = np.tanh(h1 @ a2.T + c2)
    z = h2 @ v3 + c3
    r = softplus(z) - y
    loss = float(np.mean(r * r))
    dz = 2.0 * r / n / (1.0 + np.exp(-z))
    d2 = (dz[:, None] * v3[None, :]) * (1.0 - h2 * h2)
    d1 = (d2 @ a2) * (1.0 - h1 * h1)
    g = np.zeros(NPARAM)
    g[W1:B1] = (d1.T @ x).reshape(-1)
    g[B1:W2] = d1.sum(0)
    g[W2:B2] = (d2.T @ h1).reshape(-1)
    g[B2:W3] = d2.sum(0)
    g[W3:B3] = h2.T @ dz
    g[B3] = dz.sum()
    return loss, g


def adam(w, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (Kingma & Ba 2015), in place; returns w."""
    m[:] = b1 * m + (1 - b1) * g
    v[:] = b2 * v + (1 - b2) * g * g
    w -= lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return w


def xavier_init(seed=0):
    """Xavier-uniform weights, zero biases (the same as the package's init)."""
    rng = np.random.default_rng(seed)
    w = np.zeros(NPARAM)
    for lo, fan_in, fan_out in ((W1, NIN, NHID), (W2, NHID, NHID), (W3, NHID, 1)):
        lim = np.sqrt(6.0 / (fan_in + fan_out))
        w[lo:lo + fan_in * fan_out] = rng.uniform(-lim, lim, fan_in * fan_out)
    return w


def node_features(f, rho, ux, uy, tau0):
    """Features of nodes from their post-stream populations f[9][...]:
    rho, |u|, Pi/|Pi| (xx, xy, yy), |S|, with Pi = sum e e (f - feq) and
    S = -3/(2 rho tau0) Pi."""
    ex = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1], dtype=np.float64)
    ey = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1], dtype=np.float64)
    wk = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
    f = np.asarray(f, dtype=np.float64)
    shp = (9,) + (1,) * (f.ndim - 1)
    eu = ex.reshape(shp) * ux + ey.reshape(shp) * uy
    feq = wk.reshape(shp) * rho * (1 + 3 * eu + 4.5 * eu * eu - 1.5 * (ux * ux + uy * uy))
    d = f - feq
    pxx = np.sum((ex * ex).reshape(shp) * d, 0)
    pxy = np.sum((ex * ey).reshape(shp) * d, 0)
    pyy = np.sum((ey * ey).reshape(shp) * d, 0)
    c = -1.5 / (rho * tau0)
    pn = np.sqrt(pxx * pxx + 2 * pxy * pxy + pyy * pyy)
    inv = np.where(pn > 0, 1.0 / np.where(pn > 0, pn, 1.0), 0.0)
    smag = np.sqrt(2 * ((pxx * c) ** 2 + 2 * (pxy * c) ** 2 + (pyy * c) ** 2))
    return np.stack([rho, np.sqrt(ux * ux + uy * uy), pxx * inv, pxy * inv, pyy * inv, smag], -1)
