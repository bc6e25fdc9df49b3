"""Oracle for the tree updates between rebuilds: a numpy restatement of
Gravity_Tree_Update_Kicks and Gravity_Tree_Update_Drift
(src/Gravity/tree_update.c:12-104) in the reference's Float / float / double
order.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path (tests/ import it).
It is pinned against the reference itself (ref_harness mode "update",
tests/test_oracle_tree_update.py).

Between two domain decompositions the reference keeps its tree. Every kick of
an active particle (kick.c:31-32, 61-62) adds its momentum change, divided by
the node mass, to Dp of every subtree node from Tree_Parent up to (not
including) the subtree's first node, which carries the TOP flag, and then to
its top node, which it marks by a negative Level. The drift (drift.c:41-42)
moves every marked node by Time.Step * Dp and clears Dp and the marks.
"""
from __future__ import annotations

import numpy as np

TOP = 1 << 10        # Tree_Bitfield TOP (tree.h:64)
UPDATED = 1 << 11    # Tree_Bitfield UPDATED


def _ft(fsize):
    return np.float32 if fsize == 4 else np.float64


def particle_dp(mass, dt, acc, fsize):
    """dp of tree_update.c:14-17: m_dt = Float(Mass * (double) dt), then
    m_dt * Acc in Float. mass, dt: (n,), acc: (3, n)."""
    F = _ft(fsize)
    m_dt = (np.asarray(mass, F).astype(np.float64) * np.asarray(dt, F).astype(np.float64)).astype(F)
    return (m_dt[None, :] * np.asarray(acc, F)).astype(F)


def kicks(tree, top, tree_parent, order, dp, fsize):
    """Gravity_Tree_Update_Kicks (tree_update.c:12-54) for the particles in
    `order` (the Active_Particle_List, as one thread runs it), dp[:, i] the
    Float momentum change of particle i (particle_dp). Returns updated
    copies of tree and top."""
    F = _ft(fsize)
    tree, top = tree.copy(), top.copy()
    bf, dup, tmass, tdp = tree["Bitfield"], tree["DUp"], tree["Mass"], tree["Dp"]
    for i in order:
        d = [F(dp[0, i]), F(dp[1, i]), F(dp[2, i])]
        node = int(tree_parent[i])
        if node >= 0:
            while not (bf[node] & TOP):
                m = tmass[node]
                for k in range(3):
                    tdp[node, k] = F(tdp[node, k] + F(d[k] / m))
                bf[node] |= UPDATED
                node -= int(dup[node])
            t = int(dup[node])
        else:
            t = -node - 1
        if top["Level"][t] > 0:
            top["Level"][t] *= -1
        tm = top["Mass"][t]
        for k in range(3):
            if fsize == 4:
                top["Dp"][t, k] = np.float32(top["Dp"][t, k] + np.float32(d[k] / tm))
            else:
                top["Dp"][t, k] = np.float32(np.float64(top["Dp"][t, k])
                                             + np.float64(d[k]) / np.float64(tm))
    return tree, top


def drift(tree, top, dt, fsize):
    """Gravity_Tree_Update_Drift (tree_update.c:62-101): CoM += dt * Dp (in
    double, rounded to the node's type) for marked nodes, then Dp = 0 and the
    marks cleared. Returns updated copies."""
    F = _ft(fsize)
    tree, top = tree.copy(), top.copy()
    m = (tree["Bitfield"] & UPDATED) != 0
    com = tree["CoM"][m].astype(np.float64)
    tree["CoM"][m] = (com + dt * tree["Dp"][m].astype(np.float64)).astype(F)
    tree["Dp"][m] = 0
    tree["Bitfield"][m] &= ~np.uint32(UPDATED)
    t = top["Level"] < 0
    tcom = top["CoM"][t].astype(np.float64)
    top["CoM"][t] = (tcom + dt * top["Dp"][t].astype(np.float64)).astype(np.float32)
    top["Dp"][t] = 0
    top["Level"][t] *= -1
    return tree, top
