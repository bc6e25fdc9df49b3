"""Oracle for the learned Ewald correction's network (FP64 numpy restatement
of the forward pass and the gradient of the mean-square loss).

TEST INFRASTRUCTURE ONLY: checks the CUDA training kernels
(tandav_b200/csrc/tvg_ewald_mlp.cu). The reference has no learned part; the
model is T(x) = 4 pi x / 3 + W3 tanh(W2 tanh(W1 (4 x - 1) + b1) + b2) + b3 on
the folded octant, parameters packed as W1[64][3], b1, W2[64][64], b2,
W3[3][64], b3.
"""
from __future__ import annotations

import math

import numpy as np

H = 64
LIN = 4.0 * math.pi / 3.0
OFF = {"W1": 0, "b1": 3 * H, "W2": 4 * H, "b2": 4 * H + H * H, "W3": 5 * H + H * H,
       "b3": 8 * H + H * H}
NPARAM = 8 * H + H * H + 3


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[OFF["W1"]:OFF["b1"]].reshape(H, 3), p[OFF["b1"]:OFF["W2"]],
            p[OFF["W2"]:OFF["b2"]].reshape(H, H), p[OFF["b2"]:OFF["W3"]],
            p[OFF["W3"]:OFF["b3"]].reshape(3, H), p[OFF["b3"]:])


def forward(p, x):
    """T(x) for x (n, 3) on the octant (box units)."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    v = 4.0 * np.asarray(x, np.float64) - 1.0
    a1 = np.tanh(v @ W1.T + b1)
    a2 = np.tanh(a1 @ W2.T + b2)
    return LIN * np.asarray(x, np.float64) + a2 @ W3.T + b3


def grad(p, x, y):
    """Gradient of mean((net(x) - y)^2) over the n x 3 outputs, where y is the
    residual target T(x) - 4 pi x / 3; returns (grad (NPARAM,), loss sum)."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    x = np.asarray(x, np.float64)
    v = 4.0 * x - 1.0
    a1 = np.tanh(v @ W1.T + b1)
    a2 = np.tanh(a1 @ W2.T + b2)
    out = a2 @ W3.T + b3
    r = out - np.asarray(y, np.float64)
    n = x.shape[0]
    dy = 2.0 * r / (3.0 * n)
    g = np.zeros(NPARAM)
    g[OFF["W3"]:OFF["b3"]] = (dy.T @ a2).reshape(-1)
    g[OFF["b3"]:] = dy.sum(0)
    dz2 = (dy @ W3) * (1.0 - a2 * a2)
    g[OFF["W2"]:OFF["b2"]] = (dz2.T @ a1).reshape(-1)
    g[OFF["b2"]:OFF["W3"]] = dz2.sum(0)
    dz1 = (dz2 @ W2) * (1.0 - a1 * a1)
    g[OFF["W1"]:OFF["b1"]] = (dz1.T @ v).reshape(-1)
    g[OFF["b1"]:OFF["W2"]] = dz1.sum(0)
    return g, float((r * r).sum())


def trilinear(table, x):
    """The reference's interpolation (Gravity/periodic.c:35-113) of a 65^3
    octant table (box units, (fx, fy, fz) flat) at octant points x (n, 3)."""
    fx, fy, fz = (np.asarray(t).reshape(65, 65, 65) for t in table)
    u = np.asarray(x, np.float64) * 128.0
    i = np.minimum(u.astype(int), 63)
    w = u - i
    out = np.zeros((len(u), 3))
    for c, f in enumerate((fx, fy, fz)):
        acc = 0.0
        for a in (0, 1):
            for b in (0, 1):
                for d in (0, 1):
                    wt = ((w[:, 0] if a else 1 - w[:, 0]) * (w[:, 1] if b else 1 - w[:, 1])
                          * (w[:, 2] if d else 1 - w[:, 2]))
                    acc = acc + wt * f[i[:, 0] + a, i[:, 1] + b, i[:, 2] + d]
        out[:, c] = acc
    return out
