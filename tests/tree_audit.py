"""The reference's own tree audit (test_gravity_tree,
src/Gravity/tree_build.c:620-685), extended from its first ten nodes to every
node and vectorized, as a size-independent check of a built tree.

The reference walks each node's branch in pre-order until the level returns
to the node's, collects the particles of the bundles and leaves it meets, and
prints their number, mass and centre of mass beside the node's, with the
count of particles outside the node's cube. Here every node is held to:

* the branch the level walk finds ends where DNext says it does;
* its bundles and leaves hold Npart particles in one contiguous range (all
  particles are covered once, together with the top nodes without subtree);
* mass and centre of mass equal the FP64 sums over that range within the
  Float rounding of the build, and the centre of mass lies in the node's
  cube;
* each child is one level below its parent and its cube is the parent's
  octant, and each particle lies in the cube of its bundle or leaf (so in
  every ancestor's cube: the audit's "nout" is zero);
* except where the reference's own rule moves a cube: a node takes its
  centre from its first particle by the sign test `pos > parent centre`
  (tree_build.c:542-550), while the key truncates, so a first particle
  exactly on the parent's centre plane puts the node (and its descendants)
  one cell below the octant its key, and so its particles, belong to. Such
  axes are found exactly and excused; nothing else is;
* the subtree's first node repeats its top node (Npart, centre, level).

Test infrastructure only.
"""
from __future__ import annotations

import numpy as np

TOP = 1 << 10


def branch_end(level):
    """For every node, the first later node whose level is <= its own: where
    the audit's `while (Level(n) > lvl)` stops (len(level) if none)."""
    n = len(level)
    end = np.full(n, n, np.int64)
    for lv in np.unique(level):
        stop = np.flatnonzero(level <= lv)
        mine = np.flatnonzero(level == lv)
        k = np.searchsorted(stop, mine, side="right")
        ok = k < len(stop)
        end[mine[ok]] = stop[k[ok]]
    return end


def audit(tree, top, pos, mass, domain_size, fsize, vector_size=64, top_level=2):
    """Raises AssertionError naming the first failed check; returns figures."""
    nn = len(tree)
    npart_all = len(mass)
    bf = tree["Bitfield"].astype(np.int64)
    lvl = bf & 0x3F
    dn = tree["DNext"].astype(np.int64)
    cnt = tree["Npart"].astype(np.int64)
    dup = tree["DUp"].astype(np.int64)
    is_top = (bf & TOP) != 0
    leaf = dn < 0
    internal = dn > 0
    idx = np.arange(nn)
    eps = np.finfo(np.float32 if fsize == 4 else np.float64).eps

    # the level walk of the audit and the DNext skip pointers agree
    end = branch_end(lvl)
    bad = np.flatnonzero(internal & (end != idx + dn))
    assert bad.size == 0, f"branch end differs from DNext at nodes {bad[:8]}"

    # bundles and leaves: contiguous ranges covering each branch
    li = np.flatnonzero(leaf)
    start = -dn[li] - 1
    lc = cnt[li]
    assert np.all(lc > 0) and np.all(start >= 0) and np.all(start + lc <= npart_all)
    ii = np.flatnonzero(internal)
    a = np.searchsorted(li, ii, side="right")
    b = np.searchsorted(li, end[ii], side="left")
    assert np.all(b > a), "internal node without bundle or leaf"
    breaks = np.concatenate([[0], np.cumsum(start[1:] != start[:-1] + lc[:-1])])
    bad = np.flatnonzero(breaks[b - 1] != breaks[a])
    assert bad.size == 0, f"branch particles not contiguous at nodes {ii[bad[:8]]}"
    first = np.empty(nn, np.int64)
    first[li] = start
    first[ii] = start[a]
    span = start[b - 1] + lc[b - 1] - start[a]
    bad = np.flatnonzero(span != cnt[ii])
    assert bad.size == 0, f"Npart differs from the branch's particles at nodes {ii[bad[:8]]}"

    # every particle once: leaves plus the top nodes without subtree
    cover = np.zeros(npart_all + 1, np.int64)
    np.add.at(cover, start, 1)
    np.add.at(cover, start + lc, -1)
    small = top["Npart"] <= vector_size
    np.add.at(cover, top["First_Part"][small].astype(np.int64), 1)
    np.add.at(cover, (top["First_Part"][small] + top["Npart"][small]).astype(np.int64), -1)
    assert np.array_equal(np.cumsum(cover)[:npart_all], np.ones(npart_all, np.int64)), \
        "particles not covered exactly once"

    # mass and centre of mass against FP64 sums over the node's range
    m64 = np.asarray(mass, np.float64)
    x64 = np.asarray(pos, np.float64)
    S = np.concatenate([[0.0], np.cumsum(m64)])
    SX = [np.concatenate([[0.0], np.cumsum(m64 * x64[k])]) for k in range(3)]
    nodes = np.flatnonzero(leaf | internal)
    lo, hi = first[nodes], first[nodes] + cnt[nodes]
    M = S[hi] - S[lo]
    m_err = np.abs(M - tree["Mass"][nodes].astype(np.float64)) / M
    c_err = np.zeros(len(nodes))
    for k in range(3):
        com = (SX[k][hi] - SX[k][lo]) / M
        c_err = np.maximum(c_err, np.abs(com - tree["CoM"][nodes, k].astype(np.float64))
                           / np.maximum(np.abs(com), domain_size))
    # the centre of mass of particles in a cube lies in the cube
    nsize = domain_size / (2.0 ** lvl[nodes])
    c_out = np.abs(tree["CoM"][nodes].astype(np.float64) - tree["Pos"][nodes].astype(np.float64)) \
        - nsize[:, None] / 2

    # geometry: octant of the parent, particles inside their leaf's cube
    inner = np.flatnonzero((leaf | internal) & ~is_top)
    par = inner - dup[inner]
    assert np.all(par >= 0) and np.all(internal[par]), "parent is not an internal node"
    assert np.array_equal(lvl[inner], lvl[par] + 1), "child not one level below its parent"
    half = domain_size / (2.0 ** lvl[inner]) / 2
    off = np.abs(tree["Pos"][inner].astype(np.float64) - tree["Pos"][par].astype(np.float64))
    g_err = np.abs(off - half[:, None]).max() / domain_size if inner.size else 0.0
    # axes on which a node's cube is moved by a first particle on its parent's
    # centre plane, inherited by the descendants (parents precede children)
    ft = np.float32 if fsize == 4 else np.float64
    pos_f = np.asarray(pos, ft)
    shifted = np.zeros((nn, 3), bool)
    fp = first[inner]
    own = (pos_f[:, fp].T == tree["Pos"][par]) & (tree["Pos"][inner] < tree["Pos"][par])
    order = np.argsort(lvl[inner], kind="stable")
    for lv in np.unique(lvl[inner]):
        sel = order[lvl[inner][order] == lv]
        shifted[inner[sel]] = own[sel] | shifted[par[sel]]
    owner = np.repeat(li, lc)
    pidx = np.repeat(start - (np.cumsum(lc) - lc), lc) + np.arange(int(lc.sum()))
    lsize = domain_size / (2.0 ** lvl[owner])
    out = np.abs(x64[:, pidx].T - tree["Pos"][owner].astype(np.float64)) - lsize[:, None] / 2
    nout = int((out > 0).all(1).sum())            # the reference's count
    out = np.where(shifted[owner], 0.0, out)
    p_err = max(0.0, out.max() / domain_size) if out.size else 0.0

    c_out = np.where(shifted[nodes], 0.0, c_out)
    c_out = max(0.0, c_out.max() / domain_size) if nodes.size else 0.0

    # subtree roots repeat their top nodes
    roots = np.flatnonzero(is_top & internal)
    t = dup[roots]
    assert np.array_equal(cnt[roots], top["Npart"][t].astype(np.int64))
    assert np.array_equal(lvl[roots], np.full(len(roots), top_level))
    assert np.array_equal(tree["Pos"][roots].astype(np.float32), top["Pos"][t])

    figures = dict(nodes=int(len(nodes)), mass_rel=float(m_err.max()), com_rel=float(c_err.max()),
                   com_outside_rel=float(c_out), octant_rel=float(g_err), outside_rel=float(p_err),
                   nout=nout, moved_nodes=int(shifted.any(1).sum()))
    assert nout == 0, figures
    # Float sums in the build's order: bounds in units of the Float epsilon;
    # node centres descend from the top nodes' float centres (domain.h:47)
    # in both builds, so the geometry is held to the float epsilon
    feps = np.finfo(np.float32).eps
    assert figures["mass_rel"] < 256 * eps * max(1.0, np.sqrt(npart_all)), figures
    assert figures["com_rel"] < 256 * eps * max(1.0, np.sqrt(npart_all)), figures
    assert figures["octant_rel"] < 64 * feps, figures
    assert figures["outside_rel"] < 64 * feps, figures
    assert figures["com_outside_rel"] < 64 * feps, figures
    return figures
