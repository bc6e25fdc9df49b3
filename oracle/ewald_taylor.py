"""CPU restatement of the group form's Taylor table of the Ewald correction
(tandav_b200/csrc/tvg_ewald.cu: k_ewald_fine, k_ewald_taylor; the lookup in
tandav_b200/csrc/tvg_walk_group.cu: ewald_kjh_taylor).

TEST INFRASTRUCTURE ONLY: it checks the scheme (finite differences on a
grid of half the node spacing, third-order expansion about the nearest node)
against direct lattice sums. The sums come from the oracle's restatement of
compute_ewald_force (Gravity/periodic.c:352-461), which is pinned against
the reference's own table. The reference has no Taylor table.

Record layout, 20 values per component a (node units u = 2 (N - 1) x):
[0] T_a, [1 + b] dT_a/du_b, [4 + s] d2T_a for s in xx yy zz xy xz yz,
[10 + t] d3T_a for t in xxx yyy zzz xxy xxz yyx yyz zzx zzy xyz.
"""
from __future__ import annotations

import numpy as np

import port

PAIRS = [(0, 1), (0, 2), (1, 2)]
BBE = [(0, 1), (0, 2), (1, 0), (1, 2), (2, 0), (2, 1)]


def record(node, nodes=33):
    """The 60 values of the table record at integer node (i, j, k), FP64
    finite differences rounded to FP32 as the table stores them."""
    d = 1.0 / (4.0 * (nodes - 1))               # fine spacing, box units
    offs = np.array([(a, b, c) for a in range(-2, 3) for b in range(-2, 3) for c in range(-2, 3)])
    x = (2 * np.asarray(node) + offs) * d
    f = port.ewald_force(x)
    F = {tuple(o): f[n] for n, o in enumerate(offs)}
    h = 0.5                                      # fine spacing, node units
    out = np.zeros(60)
    for a in range(3):
        r = out[20 * a:20 * a + 20]

        def g(b, s):
            o = [0, 0, 0]
            o[b] = s
            return F[tuple(o)][a]

        def g2(b, sb, e, se):
            o = [0, 0, 0]
            o[b] += sb
            o[e] += se
            return F[tuple(o)][a]

        c = F[(0, 0, 0)][a]
        r[0] = c
        for b in range(3):
            r[1 + b] = (-g(b, 2) + 8 * g(b, 1) - 8 * g(b, -1) + g(b, -2)) / (12 * h)
            r[4 + b] = (-g(b, 2) + 16 * g(b, 1) - 30 * c + 16 * g(b, -1) - g(b, -2)) / (12 * h * h)
            r[10 + b] = (g(b, 2) - 2 * g(b, 1) + 2 * g(b, -1) - g(b, -2)) / (2 * h ** 3)
        for q, (b, e) in enumerate(PAIRS):
            r[7 + q] = (g2(b, 1, e, 1) - g2(b, 1, e, -1) - g2(b, -1, e, 1) + g2(b, -1, e, -1)) / (4 * h * h)
        for q, (b, e) in enumerate(BBE):
            up = g2(b, 1, e, 1) - 2 * g2(b, 0, e, 1) + g2(b, -1, e, 1)
            dn = g2(b, 1, e, -1) - 2 * g2(b, 0, e, -1) + g2(b, -1, e, -1)
            r[13 + q] = (up - dn) / (2 * h ** 3)
        r[19] = sum(sx * sy * sz * F[(sx, sy, sz)][a] for sx in (-1, 1) for sy in (-1, 1)
                    for sz in (-1, 1)) / (8 * h ** 3)
    return out.astype(np.float32).astype(np.float64)


def evaluate(rec, du):
    """T, dT/du and d2T/du du at node + du (node units), as the lookup
    expands them: with D = d3T . du, T + du . (dT + (d2T + D/3) du / 2),
    dT + (d2T + D/2) du and d2T + D."""
    du = np.asarray(du, np.float64)
    val, grad, hess = np.zeros(3), np.zeros((3, 3)), np.zeros((3, 3, 3))
    for a in range(3):
        r = rec[20 * a:20 * a + 20]
        H = np.empty((3, 3))
        for b in range(3):
            H[b, b] = r[4 + b]
        for q, (b, e) in enumerate(PAIRS):
            H[b, e] = H[e, b] = r[7 + q]
        T3 = np.empty((3, 3, 3))
        pure = {0: r[10], 1: r[11], 2: r[12]}
        for b in range(3):
            T3[b, b, b] = pure[b]
        for q, (b, e) in enumerate(BBE):
            for idx in ((b, b, e), (b, e, b), (e, b, b)):
                T3[idx] = r[13 + q]
        for idx in ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)):
            T3[idx] = r[19]
        D = T3 @ du
        hess[a] = H + D
        grad[a] = r[1:4] + (H + D / 2) @ du
        val[a] = r[0] + du @ (r[1:4] + 0.5 * ((H + D / 3) @ du))
    return val, grad, hess
