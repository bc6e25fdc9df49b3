"""The group form (FP32 integer-offset, warp per PH group): force accuracy
against FP64 direct summation (Ewald-summed in the periodic box) with the
reference's softened kernel, and agreement with the plain form.

Tolerances: the relative criterion at errtol 0.005 gives rms relative errors
~1e-3 in the reference (its own walk, run on small boxes); the group tests
are conservative for the whole group, so their rms error must stay at or
below the plain form's (with 20 % slack) and below 1e-3 where the plain form
is below it."""
import numpy as np
import pytest

import port
from tandav_b200 import gravity as G
from tandav_b200 import ics

pytestmark = pytest.mark.gpu

_CORR = {}


def fine_corr_table():
    """FP64 correction on the 65^3 octant grid, interleaved (x, y, z)."""
    if "t" not in _CORR:
        fx, fy, fz, _ = port.ewald_table(64)
        _CORR["t"] = np.stack([fx, fy, fz], axis=1).reshape(-1).copy()
    return _CORR["t"]


def rel_err(a, ref):
    d = np.sqrt(((a - ref) ** 2).sum(0))
    return d / np.sqrt((ref ** 2).sum(0))


def run_walks(p, origin, size, form, fsize=4, flags=0, open_rel=0.005):
    periodic = p.box > 0
    parts = G.WALK_GRAVITY | (G.WALK_EWALD if periodic else 0)
    with G.GravityContext(max(p.n, 1024), float_bytes=fsize, periodic=periodic, boxsize=p.box,
                          softening=p.softening, flags=flags, open_rel=open_rel) as ctx:
        ctx.upload(p.pos, p.mass)
        ctx.set_domain(origin, size)
        ctx.peano_keys()
        perm = ctx.sort_particles()
        ctx.top_nodes()
        ctx.tree_build(exact_moments=(form == G.FORM_PLAIN))
        if periodic:
            ctx.ewald_init()
        ctx.zero_accel()
        ctx.walk(form, use_bh=True, parts=parts)
        bh = ctx.download(G.F_GRAV_ACC | G.F_COST)
        counts = {"bh": ctx.walk_counters() + (ctx.walk_quad_interactions(),)}
        ctx.save_last_accel()
        ctx.walk(form, use_bh=False, parts=parts)
        rel = ctx.download(G.F_GRAV_ACC | G.F_COST)
        counts["rel"] = ctx.walk_counters() + (ctx.walk_quad_interactions(),)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(perm))
    out = {k: (v["grav_acc"][:, inv].astype(np.float64), v["cost"][inv]) for k, v in
           (("bh", bh), ("rel", rel))}
    out["counts"] = counts
    return out


def _case(kind):
    if kind == "hernquist":
        p = ics.hernquist(n=32768, seed=31)
        c = np.median(p.pos, axis=1)
        size = 2.001 * np.abs(p.pos - c[:, None]).max()
        return p, c - 0.5 * size, size, None
    p = ics.zeldovich_box(n_side=32, seed=32)
    return p, np.zeros(3), p.box, fine_corr_table()


@pytest.mark.parametrize("kind", ["hernquist", "zeldovich"])
def test_group_accuracy(kind):
    p, origin, size, corr = _case(kind)
    rng = np.random.default_rng(5)
    tgt = rng.choice(p.n, 1000, replace=False)
    ref = port.direct(p.pos, p.mass, tgt, ics.GRAVITY, p.softening, box=p.box,
                      corr_table=corr, corr_n=64)
    plain = run_walks(p, origin, size, G.FORM_PLAIN)
    group = run_walks(p, origin, size, G.FORM_GROUP)
    for crit in ("bh", "rel"):
        ep = rel_err(plain[crit][0][:, tgt], ref)
        eg = rel_err(group[crit][0][:, tgt], ref)
        rms_p, rms_g = np.sqrt((ep ** 2).mean()), np.sqrt((eg ** 2).mean())
        print(f"{kind} {crit}: rms plain {rms_p:.3e} group {rms_g:.3e}; "
              f"p99 plain {np.percentile(ep, 99):.3e} group {np.percentile(eg, 99):.3e}; "
              f"interactions plain {plain[crit][1].mean():.0f} group {group[crit][1].mean():.0f}")
        assert rms_g <= 1.2 * rms_p + 1e-6
        if rms_p < 1e-3:
            assert rms_g < 1e-3


@pytest.mark.parametrize("kind,fsize", [("hernquist", 4), ("hernquist", 8), ("zeldovich", 4)])
def test_quadrupole_accuracy(kind, fsize):
    """TVG_CFG_QUADRUPOLE (no reference counterpart): under the BH criterion
    the walk accepts the same nodes as the monopole walk, so the interaction
    counts are equal, and every accepted node's quadrupole lowers the error.
    Under the relative criterion (octupole-order bound), in the isolated halo
    the error at the same TREE_OPEN_PARAM_REL is lower with fewer
    interactions. The 32^3 Zel'dovich box at z = 50 is nearly a perfect
    lattice, whose cubic nodes have no quadrupole (nor octupole) moment: the
    error there is the next order, which the looser criterion lets grow, and
    the quadrupole walk needs a quarter of the monopole walk's parameter for
    the same error."""
    p, origin, size, corr = _case(kind)
    tgt = np.random.default_rng(5).choice(p.n, 1000, replace=False)
    ref = port.direct(p.pos, p.mass, tgt, ics.GRAVITY, p.softening, box=p.box,
                      corr_table=corr, corr_n=64)
    mono = run_walks(p, origin, size, G.FORM_GROUP, fsize=fsize)
    quad = run_walks(p, origin, size, G.FORM_GROUP, fsize=fsize, flags=G.CFG_QUADRUPOLE,
                     open_rel=0.005 if p.box == 0 else 0.005 / 4)
    for crit in ("bh", "rel"):
        em = rel_err(mono[crit][0][:, tgt], ref)
        eq = rel_err(quad[crit][0][:, tgt], ref)
        rms_m, rms_q = np.sqrt((em ** 2).mean()), np.sqrt((eq ** 2).mean())
        (gm, ewm, qm), (gq, ewq, qq) = mono["counts"][crit], quad["counts"][crit]
        print(f"{kind} f{fsize} {crit}: rms monopole {rms_m:.3e} quadrupole {rms_q:.3e}; "
              f"interactions {gm / p.n:.0f} / {gq / p.n:.0f} (quadrupole {qq / p.n:.0f})")
        assert qm == 0 and 0 < qq < gq
        if crit == "bh":
            assert gq == gm and ewq == ewm
            # (in the periodic box the Ewald walk's own monopole error stays)
            assert rms_q < (0.5 if p.box == 0 else 0.8) * rms_m
        elif p.box == 0:
            assert gq < gm
            assert rms_q < rms_m and rms_q < 1e-3
        else:
            assert rms_q < rms_m


def _periodic_walk(p, flags, open_rel, ewald_alpha, tgt, ntask=1, cost=None, tops=None):
    parts = G.WALK_GRAVITY | G.WALK_EWALD
    with G.GravityContext(p.n, float_bytes=4, periodic=True, boxsize=p.box, softening=p.softening,
                          flags=flags) as ctx:
        if ntask > 1:
            ctx.set_domain_decomposition(ntask)
        ctx.upload(p.pos, p.mass, cost=cost)
        ctx.set_domain((0.0, 0.0, 0.0), p.box)
        ctx.ewald_init()
        ctx.set_ewald_opening(ewald_alpha)
        ctx.force_step(form=G.FORM_GROUP, use_bh=True, parts=parts)
        ctx.save_last_accel()
        ctx.set_opening(0.25, open_rel)
        ctx.force_step(form=G.FORM_GROUP, use_bh=False, parts=parts)
        counts = ctx.walk_counters() + (ctx.walk_quad_interactions(),)
        if tops is not None:
            tops.append(len(ctx.download_tree()[1]))
        ids = ctx.download(G.F_ID)["id"]
        inv = np.empty(p.n, np.int64)
        inv[ids] = np.arange(p.n)
        _, _, err = ctx.forcetest(np.sort(inv[tgt]))
    return err, counts


def test_quadrupole_periodic_with_centre_images():
    """A 64^3 Zel'dovich box, where the groups take the image nearest to
    their centre: the quadrupole walk (gravity and Ewald walks) at the same
    TREE_OPEN_PARAM_REL is more accurate than the monopole walk with fewer
    gravity and Ewald interactions, and below 1e-3 rms (FP64 direct Ewald sum
    on the GPU, tvg_forcetest)."""
    p = ics.zeldovich_box(n_side=64, seed=33)
    tgt = np.random.default_rng(6).choice(p.n, 4000, replace=False)
    err_m, (gm, em, qm) = _periodic_walk(p, 0, 3e-3, 1e-2, tgt)
    err_q, (gq, eq, qq) = _periodic_walk(p, G.CFG_QUADRUPOLE, 3e-3, 1e-2, tgt)
    print(f"64^3: rms monopole {err_m['rms']:.3e} quadrupole {err_q['rms']:.3e}; gravity "
          f"{gm / p.n:.0f} / {gq / p.n:.0f} (quadrupole {qq / p.n:.0f}); Ewald {em / p.n:.1f} / "
          f"{eq / p.n:.1f}")
    assert qm == 0 and 0 < qq < gq
    assert gq < gm and eq < em
    assert err_q["rms"] < err_m["rms"] and err_q["rms"] < 1e-3


def test_walk_limit_times_out_and_the_context_recovers():
    """The group walks' traversal loops are bounded (tvg_set_walk_limit): with
    a limit of two iterations the gravity and Ewald walks (which a periodic
    group walk runs together) stop, tvg_walk returns TVG_E_TIMEOUT, and the
    context stays usable -- with the limit restored the same walk gives the
    accelerations of a walk that never timed out. An isolated context stops
    its gravity walk the same way."""
    # 32^3: 512 particles per level-2 cell, so every top node has a subtree
    # and a group needs many node batches
    p = ics.zeldovich_box(n_side=32, seed=34)
    parts = G.WALK_GRAVITY | G.WALK_EWALD
    with G.GravityContext(p.n, float_bytes=4, periodic=True, boxsize=p.box,
                          softening=p.softening) as ctx:
        ctx.upload(p.pos, p.mass)
        ctx.set_domain((0.0, 0.0, 0.0), p.box)
        ctx.peano_keys()
        ctx.sort_particles()
        ctx.top_nodes()
        ctx.tree_build()
        ctx.ewald_init()
        ctx.zero_accel()
        ctx.walk(G.FORM_GROUP, use_bh=True, parts=parts)
        first = ctx.download(G.F_GRAV_ACC)["grav_acc"].copy()
        ctx.set_walk_limit(2)
        ctx.zero_accel()
        with pytest.raises(G.TvgError) as e:
            ctx.walk(G.FORM_GROUP, use_bh=True, parts=parts)
        assert e.value.code == 4, e.value          # TVG_E_TIMEOUT
        ctx.set_walk_limit()
        ctx.zero_accel()
        ctx.walk(G.FORM_GROUP, use_bh=True, parts=parts)
        assert np.array_equal(ctx.download(G.F_GRAV_ACC)["grav_acc"], first)
    h = ics.hernquist(n=32768, seed=37)
    c = np.median(h.pos, axis=1)
    size = 2.001 * float(np.abs(h.pos - c[:, None]).max())
    with G.GravityContext(h.n, float_bytes=4, softening=h.softening) as ctx:
        ctx.upload(h.pos, h.mass)
        ctx.set_domain(c - 0.5 * size, size)
        ctx.peano_keys()
        ctx.sort_particles()
        ctx.top_nodes()
        ctx.tree_build()
        ctx.set_walk_limit(2)
        ctx.zero_accel()
        with pytest.raises(G.TvgError) as e:
            ctx.walk(G.FORM_GROUP, use_bh=True, parts=G.WALK_GRAVITY)
        assert e.value.code == 4, e.value


def test_autotune_on_a_sample_leaves_the_active_set_and_the_chosen_walk():
    """tvg_autotune times the three group sizes on a sample (every 8th window
    of 128 active particles), then walks the whole active set with the
    fastest: the accelerations it leaves equal a later walk with the same
    choice, for all particles and for an active list, whose length the
    sample must not change."""
    p = ics.zeldovich_box(n_side=32, seed=35)
    parts = G.WALK_GRAVITY | G.WALK_EWALD
    with G.GravityContext(p.n, float_bytes=4, periodic=True, boxsize=p.box,
                          softening=p.softening) as ctx:
        ctx.upload(p.pos, p.mass)
        ctx.set_domain((0.0, 0.0, 0.0), p.box)
        ctx.peano_keys()
        ctx.sort_particles()
        ctx.top_nodes()
        ctx.tree_build()
        ctx.ewald_init()
        for active in (None, np.arange(0, p.n, 3, dtype=np.int32)):
            ctx.set_active(active)
            ctx.zero_accel()
            choice, ms = ctx.autotune(use_bh=True, parts=parts)
            assert choice in (1, 2, 4) and all(t > 0 for t in ms)
            tuned = ctx.download(G.F_GRAV_ACC | G.F_ACC)
            ctx.zero_accel()
            ctx.walk(G.FORM_GROUP, use_bh=True, parts=parts)
            again = ctx.download(G.F_GRAV_ACC | G.F_ACC)
            assert np.array_equal(tuned["grav_acc"], again["grav_acc"])
            # Acc holds one walk's contribution, not the trial walks' too
            assert np.array_equal(tuned["acc"], again["acc"])
            again = again["grav_acc"]
            sel = np.arange(p.n) if active is None else active
            assert np.all(np.abs(again[:, sel]).sum(0) > 0)


def test_quadrupole_with_many_top_nodes():
    """A cost-balanced decomposition over 8 targets gives a clumped box
    hundreds of top nodes, which the walks push in chunks of 256; their
    quadrupoles come from the top nodes' own particle ranges. With the same
    |a_old| (from one Barnes-Hut pass) the relative walk's force error
    against the FP64 direct Ewald sum stays that of the default top nodes."""
    p = ics.random_box(1 << 17, box=1000.0, seed=45, clumps=11)
    h = np.arange(p.n, dtype=np.uint64) * 2654435761
    cost = np.where(p.pos[0] < 120.0, 50000 - (h % 1000), h % 100 + 1).astype(np.float64)
    tgt = np.random.default_rng(7).choice(p.n, 3000, replace=False)
    parts = G.WALK_GRAVITY | G.WALK_EWALD
    kw = dict(float_bytes=4, periodic=True, boxsize=p.box, softening=p.softening,
              flags=G.CFG_QUADRUPOLE)
    with G.GravityContext(p.n, **kw) as ctx:
        ctx.upload(p.pos, p.mass)
        ctx.set_domain((0.0, 0.0, 0.0), p.box)
        ctx.force_step(form=G.FORM_GROUP, use_bh=True, parts=parts)
        d = ctx.download(G.F_GRAV_ACC | G.F_ID)
    last = np.empty(p.n)
    last[d["id"]] = np.sqrt((d["grav_acc"].astype(np.float64) ** 2).sum(0))
    out = []
    for ntask in (1, 8):
        with G.GravityContext(p.n, **kw) as ctx:
            if ntask > 1:
                ctx.set_domain_decomposition(ntask)
            ctx.upload(p.pos, p.mass, cost=cost, last_acc=last)
            ctx.set_domain((0.0, 0.0, 0.0), p.box)
            ctx.set_opening(0.25, 8e-3)
            ctx.set_ewald_opening(1e-2)
            ctx.force_step(form=G.FORM_GROUP, use_bh=False, parts=parts)
            q = ctx.walk_quad_interactions()
            ntop = len(ctx.download_tree()[1])
            ids = ctx.download(G.F_ID)["id"]
            inv = np.empty(p.n, np.int64)
            inv[ids] = np.arange(p.n)
            _, _, err = ctx.forcetest(np.sort(inv[tgt]))
        out.append((ntop, err["rms"], q))
    print(f"top nodes, rms, quadrupole interactions per particle: "
          f"{[(t, f'{e:.3e}', round(q / p.n)) for t, e, q in out]}")
    (t1, e1, _), (t8, e8, q8) = out
    assert t8 > 256 and t8 > 4 * t1 and q8 > 0
    assert e8 < 1.3 * e1 and e8 < 2e-3
