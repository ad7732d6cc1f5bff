"""NumPy restatement of the p*-seed network (test infrastructure only).

It mirrors the device network of the B200 package: 6 -> 64 -> 64 -> 1, tanh
hidden layers, BF16 rounding (round to nearest even) of the inputs of the two
tensor-core layers (features, W1, hidden activations, W2) with wide
accumulation, an FP32-weight output layer, and the straight-through backward
pass of the training kernels (gradients with the unrounded activations and
master weights).  Used to check the GPU forward and gradients, and (with
``bf16=False``) checked itself against finite differences.
"""
from __future__ import annotations

import numpy as np

NPARAM = 64 * 6 + 64 + 64 * 64 + 64 + 64 + 1


def unpack(p):
    p = np.asarray(p, np.float64)
    o = 0
    W1 = p[o:o + 384].reshape(64, 6); o += 384
    b1 = p[o:o + 64]; o += 64
    W2 = p[o:o + 4096].reshape(64, 64); o += 4096
    b2 = p[o:o + 64]; o += 64
    w3 = p[o:o + 64]; o += 64
    b3 = p[o]
    return W1, b1, W2, b2, w3, b3


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    a = np.ascontiguousarray(x, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward(p, X, bf=True):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    X = np.asarray(X, np.float64)
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    Z1 = r(X) @ r(W1).T + b1
    H1 = np.tanh(Z1)
    Z2 = r(H1) @ r(W2).T + b2
    H2 = np.tanh(Z2)
    y = H2 @ w3 + b3
    return y, (X, H1, H2)


def loss_and_grad(p, X, Y, bf=True):
    W1, b1, W2, b2, w3, b3 = unpack(p)
    y, (X, H1, H2) = forward(p, X, bf)
    n = len(Y)
    e = y - np.asarray(Y, np.float64)
    loss = float(np.sum(e * e) / n)
    dy = 2.0 * e / n
    gw3 = H2.T @ dy
    gb3 = dy.sum()
    dZ2 = dy[:, None] * w3[None, :] * (1.0 - H2 * H2)
    gW2 = dZ2.T @ H1
    gb2 = dZ2.sum(axis=0)
    dZ1 = (dZ2 @ W2) * (1.0 - H1 * H1)
    gW1 = dZ1.T @ X
    gb1 = dZ1.sum(axis=0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gw3, [gb3]])
    return loss, g


GATE = 0.2


def features(prim, gam=1.4):
    """Normalised features and the base pressure (PVRS, floored at 1e-3 pbar) of
    primitive interface states (n, 6)."""
    prim = np.asarray(prim, np.float64)
    rl, ul, pl, rr, ur, pr = prim.T
    rb, pb = 0.5 * (rl + rr), 0.5 * (pl + pr)
    cb = np.sqrt(pb / rb)
    X = np.stack([rl / rb, ul / cb, pl / pb, rr / rb, ur / cb, pr / pb], axis=1)
    al, ar = np.sqrt(gam * pl / rl), np.sqrt(gam * pr / rr)
    ppv = pb - 0.125 * (ur - ul) * (rl + rr) * (al + ar)
    return X, np.maximum(ppv, 1e-3 * pb)


def gated(X):
    """Interfaces whose wave strength |dp|/pbar + |du|/cbar exceeds the gate."""
    return np.abs(X[:, 5] - X[:, 2]) + np.abs(X[:, 4] - X[:, 1]) > GATE
