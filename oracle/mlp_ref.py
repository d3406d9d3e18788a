"""Test infrastructure, not product code: float64 numpy forward pass, MSE loss
and hand-derived gradient of the learned absorbing layers' per-face networks
(ni inputs, two tanh layers of nh, no linear outputs -- 51/32/5 in 2D,
33/32/9 in 3D; parameter block W1 b1 W2 b2 W3 b3), the CPU reference for the
GPU training kernels."""
from __future__ import annotations

import numpy as np


def unpack(p, ni, nh, no=5):
    p = np.asarray(p, np.float64)
    o = 0
    out = []
    for shape in ((nh, ni), (nh,), (nh, nh), (nh,), (no, nh), (no,)):
        k = int(np.prod(shape))
        out.append(p[o:o + k].reshape(shape))
        o += k
    return out


def forward(p, X, ni, nh, no=5):
    W1, b1, W2, b2, W3, b3 = unpack(p, ni, nh, no)
    h1 = np.tanh(X @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    return h2 @ W3.T + b3, h1, h2


def loss_and_grad(p, X, Y, ni, nh, no=5):
    """loss = mean over samples of sum_o (y_o - t_o)^2 and its gradient."""
    X = np.asarray(X, np.float64)
    Y = np.asarray(Y, np.float64)
    n = X.shape[0]
    W1, b1, W2, b2, W3, b3 = unpack(p, ni, nh, no)
    y, h1, h2 = forward(p, X, ni, nh, no)
    e = y - Y
    loss = (e ** 2).sum() / n
    dy = 2 * e / n
    dW3 = dy.T @ h2
    db3 = dy.sum(0)
    g2 = (dy @ W3) * (1 - h2 ** 2)
    dW2 = g2.T @ h1
    db2 = g2.sum(0)
    g1 = (g2 @ W2) * (1 - h1 ** 2)
    dW1 = g1.T @ X
    db1 = g1.sum(0)
    return loss, np.concatenate([a.reshape(-1) for a in (dW1, db1, dW2, db2, dW3, db3)])
