"""numpy restatement of the selector network, for checking the CUDA kernels.

TEST INFRASTRUCTURE ONLY (imported by tests/).  The reference has no learned
component: its tuning is compile-time macros (dgemm_tune.h:6-15,
sgemm_tune.h:6-15).  This file restates the library's own 7-64-64-48 ReLU MLP
with the same flat parameter layout (W1[7][64] b1 W2[64][64] b2 W3[64][48] b3)
and the same loss (mean squared error over the finite targets), so the GPU
forward pass and gradients can be compared with an independent computation.
"""
from __future__ import annotations

import numpy as np

IN, H, OUT = 7, 64, 48
SIZES = [IN * H, H, H * H, H, H * OUT, OUT]


def unpack(w: np.ndarray):
    out, o = [], 0
    for n in SIZES:
        out.append(w[o:o + n].astype(np.float64))
        o += n
    W1, b1, W2, b2, W3, b3 = out
    return W1.reshape(IN, H), b1, W2.reshape(H, H), b2, W3.reshape(H, OUT), b3


def forward(w, X):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    h1 = np.maximum(X @ W1 + b1, 0.0)
    h2 = np.maximum(h1 @ W2 + b2, 0.0)
    return h2 @ W3 + b3, (h1, h2)


def loss_and_grad(w, X, T):
    W1, b1, W2, b2, W3, b3 = unpack(w)
    X = X.astype(np.float64)
    Y, (h1, h2) = forward(w, X)
    mask = np.isfinite(T)
    cnt = max(int(mask.sum()), 1)
    D = np.where(mask, Y - np.where(mask, T, 0.0), 0.0)
    loss = float((D * D).sum() / cnt)
    dY = 2.0 * D / cnt
    gW3 = h2.T @ dY
    gb3 = dY.sum(0)
    dh2 = (dY @ W3.T) * (h2 > 0)
    gW2 = h1.T @ dh2
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ W2.T) * (h1 > 0)
    gW1 = X.T @ dh1
    gb1 = dh1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g


def features(m, n, k, ta, tb, beta0, dtype=0):
    """Same feature map as the library (tuner.cu mlp_features)."""
    m, n, k = (np.asarray(v, dtype=np.float64) for v in (m, n, k))
    return np.stack([(np.log2(m) - 7) / 3, (np.log2(n) - 7) / 3, (np.log2(k) - 7) / 3,
                     np.asarray(ta, np.float64), np.asarray(tb, np.float64),
                     np.full_like(m, float(dtype)), np.asarray(beta0, np.float64)],
                    axis=-1).astype(np.float32)
