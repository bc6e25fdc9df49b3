"""Oracle for the learned Ewald correction's network (FP64 numpy restatement
of the forward pass and the gradient of the mean-square loss).

TEST INFRASTRUCTURE ONLY: checks the CUDA training kernels
(tandav_b200/csrc/tvg_ewald_mlp.cu). The reference has no learned part; the
model on the folded octant, with v = 4 x - 1, is
    T(x) = 4 pi x / 3 + S(x) + C . m(v) + s N(v),
S the seven lattice images nearest to the octant, m the 20 monomials of
degree <= 3 (fitted coefficients C), N = W3 tanh(W2 tanh(W1 v + b1) + b2) + b3
(trained) and s its output scale; parameters packed as W1[64][3], b1,
W2[64][64], b2, W3[3][64], b3, C[3][20], s.
"""
from __future__ import annotations

import math

import numpy as np

H = 64
LIN = 4.0 * math.pi / 3.0
OFF = {"W1": 0, "b1": 3 * H, "W2": 4 * H, "b2": 4 * H + H * H, "W3": 5 * H + H * H,
       "b3": 8 * H + H * H}
NNET = 8 * H + H * H + 3
NMONO = 20
POLY = NNET
SCALE = POLY + 3 * NMONO
NPARAM = SCALE + 1


def unpack(p):
    p = np.asarray(p, np.float64)
    return (p[OFF["W1"]:OFF["b1"]].reshape(H, 3), p[OFF["b1"]:OFF["W2"]],
            p[OFF["W2"]:OFF["b2"]].reshape(H, H), p[OFF["b2"]:OFF["W3"]],
            p[OFF["W3"]:OFF["b3"]].reshape(3, H), p[OFF["b3"]:NNET])


def monomials(v):
    """The 20 monomials of degree <= 3 of v (n, 3), in the kernels' order."""
    a, b, c = v[:, 0], v[:, 1], v[:, 2]
    return np.stack([np.ones_like(a), a, b, c, a * a, a * b, a * c, b * b, b * c, c * c,
                     a ** 3, a * a * b, a * a * c, a * b * b, a * b * c, a * c * c, b ** 3,
                     b * b * c, b * c * c, c ** 3], 1)


def analytic(x):
    """4 pi x / 3 + S(x): background term and the seven nearest images."""
    x = np.asarray(x, np.float64)
    out = LIN * x
    for n in range(1, 8):
        d = x - np.array([n & 1, (n >> 1) & 1, (n >> 2) & 1], np.float64)
        r = np.sqrt((d * d).sum(1, keepdims=True))
        out = out - d / r ** 3
    return out


def forward(p, x):
    """T(x) for x (n, 3) on the octant (box units)."""
    p = np.asarray(p, np.float64)
    W1, b1, W2, b2, W3, b3 = unpack(p)
    v = 4.0 * np.asarray(x, np.float64) - 1.0
    a1 = np.tanh(v @ W1.T + b1)
    a2 = np.tanh(a1 @ W2.T + b2)
    C = p[POLY:SCALE].reshape(3, NMONO)
    return analytic(x) + monomials(v) @ C.T + p[SCALE] * (a2 @ W3.T + b3)


def grad(p, x, y):
    """Gradient of mean((N(x) - y)^2) over the n x 3 outputs, y the network's
    target; returns (grad (NPARAM,), zero on the fitted entries, loss sum)."""
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
    g[OFF["b3"]:NNET] = dy.sum(0)
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
