"""CPU oracle of the rank MLP (TEST INFRASTRUCTURE ONLY).

Float64 numpy restatement of the network the learned-rank path trains and
evaluates with its own CUDA kernels (pspaqr_public_b200/csrc/learned.cu):
x (11 standardised features) -> ReLU(W1 x + b1) (64) -> ReLU(W2 h1 + b2) (64)
-> sigmoid(w3 . h2 + b3), loss = mean over samples of (sigmoid - y)^2.
Parameter layout (flat): W1 (64 x 11, row-major), b1 (64), W2 (64 x 64,
row-major), b2 (64), w3 (64), b3 (1).  The network has no counterpart in the
reference; the oracle checks the kernels' gradients and predictions.
"""
from __future__ import annotations

import numpy as np

F, H = 11, 64
NPARAMS = H * F + H + H * H + H + H + 1


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    assert p.size == NPARAMS
    o = 0
    W1 = p[o:o + H * F].reshape(H, F); o += H * F
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    w3 = p[o:o + H]; o += H
    b3 = p[o]
    return W1, b1, W2, b2, w3, b3


def forward(p, X):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    X = np.asarray(X, dtype=np.float64)
    a1 = X @ W1.T + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0.0)
    z = h2 @ w3 + b3
    return 1.0 / (1.0 + np.exp(-z)), (X, a1, h1, a2, h2)


def loss_grad(p, X, y):
    """(loss, gradient) of mean((sigmoid - y)^2), same layout as the parameters."""
    W1, b1, W2, b2, w3, b3 = unpack(p)
    y = np.asarray(y, dtype=np.float64)
    n = len(y)
    out, (X, a1, h1, a2, h2) = forward(p, X)
    diff = out - y
    loss = float(np.sum(diff * diff) / n)
    dz = 2.0 * diff * out * (1.0 - out) / n
    gw3 = h2.T @ dz
    gb3 = dz.sum()
    d2 = np.outer(dz, w3) * (a2 > 0)
    gW2 = d2.T @ h1
    gb2 = d2.sum(0)
    d1 = (d2 @ W2) * (a1 > 0)
    gW1 = d1.T @ X
    gb1 = d1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gw3, [gb3]])
    return loss, g
