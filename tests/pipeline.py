"""Shared helpers for the tests: run the oracle restatement end to end on
one particle set and compare structured arrays field by field."""
from __future__ import annotations

import numpy as np

import port
from refrun import TOPNODE_DTYPE


def balanced_top_nodes(std_s, pos_s, cost_s, origin, size, ntask):
    """Top nodes of the reference's decomposition over `ntask` targets
    (oracle/decomposition.py), with the centres transform_bunches_into_top_nodes
    gives them (domain.c:220-250)."""
    import decomposition
    bunches, _ = decomposition.decompose(std_s[:, 0], cost_s, ntask)
    top = np.zeros(len(bunches), TOPNODE_DTYPE)
    for t, (key, level, first, npart) in enumerate(bunches):
        top[t]["Key"], top[t]["Level"], top[t]["First_Part"], top[t]["Npart"] = key, level, first, npart
        top[t]["Target"] = -1
        sz = size / float(1 << level)
        for k in range(3):
            px = float(pos_s[k, first]) - float(origin[k])
            top[t]["Pos"][k] = np.float32((np.floor(px / sz) + 0.5) * sz + float(origin[k]))
    return top


def oracle_pipeline(pos, mass, origin, size, fsize, box=0.0, softening=0.01, gravity=43007.1,
                    ewald=None, passes=("bh", "rel"), ntask=1, cost=None, vector_size=64):
    """Keys -> sort -> top nodes -> tree -> walks, as the reference runs them
    (top nodes balanced over `ntask` targets by `cost`, in input order, when
    ntask > 1; bundles of at most `vector_size` particles)."""
    ft = port.ftype(fsize)
    pos_f = np.asarray(pos).astype(ft)
    std, rev = port.peano_keys(pos_f, origin, size, fsize)
    perm = port.sort_keys(std)
    std_s, rev_s = std[perm], rev[perm]
    pos_s = pos_f[:, perm]
    mass_s = np.asarray(mass).astype(ft)[perm]
    if ntask > 1:
        top = balanced_top_nodes(std_s, pos_s, np.asarray(cost, np.float64)[perm], origin, size, ntask)
    else:
        top = port.top_nodes(std_s, pos_s, origin, size, fsize)
    tree, top, parent = port.tree_build(rev_s, pos_s, mass_s, size, top, fsize,
                                        vector_size=vector_size)
    out = dict(perm=perm, std_key=std_s, rev_key=rev_s, pos=pos_s, mass=mass_s, top=top,
               tree=tree, tree_parent=parent)
    prm = port.WalkParams(gravity=gravity, softening=softening, domain_size=size, boxsize=box,
                          open_bh=0.25, open_rel=0.005, use_bh=1, vector_size=vector_size)
    last = np.zeros(len(mass_s), ft)
    for name in passes:
        prm.use_bh = 1 if name == "bh" else 0
        g, cg = port.walk("gravity", pos_s, mass_s, last, top, tree, prm, fsize=fsize)
        gacc = g.astype(ft)
        cost = cg.astype(ft)
        if box > 0 and ewald is not None:
            e, ce = port.walk("ewald", pos_s, mass_s, last, top, tree, prm, ewald, fsize=fsize)
            out[name + "ew_gacc"] = e.astype(ft)
            out[name + "ew_cost"] = ce.astype(ft)
            gacc = (gacc.astype(np.float64) + e).astype(ft)
            cost = (cost + ce.astype(ft)).astype(ft)
        out[name + "_gacc"] = gacc
        out[name + "_cost"] = cost
        if name == "bh":
            # accel.c:28-43: |Acc| in Float becomes Last_Acc_Mag
            last = np.sqrt(gacc[0] * gacc[0] + gacc[1] * gacc[1] + gacc[2] * gacc[2]).astype(ft)
            out["last_acc_mag"] = last
    return out


def oracle_ewald_tables(fsize, box):
    """The reference's Float tables divided by Boxsize^2 (periodic.c:215-228)."""
    ft = port.ftype(fsize)
    fx, fy, fz, _ = port.ewald_table()
    return [(t.astype(ft).astype(np.float64) / (box * box)).astype(ft) for t in (fx, fy, fz)]


def assert_struct_equal(a, b, fields, what):
    assert len(a) == len(b), f"{what}: {len(a)} != {len(b)} entries"
    if len(a) == 0:
        return
    for f in fields:
        x, y = np.asarray(a[f]), np.asarray(b[f])
        bad = ~(x == y).reshape(len(a), -1).all(1)
        assert not bad.any(), f"{what}.{f} differs at {np.flatnonzero(bad)[:8]}"
