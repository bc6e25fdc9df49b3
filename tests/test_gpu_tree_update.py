"""The tree updates between rebuilds on the GPU (tvg_tree_update.cu) in the
step loop of src/main.c:43-78 with Time_For_Domain_Update, on a Hernquist
sphere (isolated) and on clumps in a periodic box (particles wrapped into
the box every drift), both filling six to eight time bins. Without a due
domain update:

* each kick adds the active particles' momentum to the kept tree: every
  node and top-node field equals the restatement (oracle/tree_update.py,
  pinned to the reference's Gravity_Tree_Update_Kicks) applied to the tree
  downloaded before the kick, with the GPU's own kick factors;
* each drift moves the kicked nodes by Time.Step * Dp, bit for bit;
* the force computation keeps the particle order and walks the updated
  tree: the plain form's accelerations equal the restatement's walk
  (port.walk) on the downloaded tree, bit for bit (gravity part; nearest
  images in the box), and (FP32, isolated) the group form on the same tree
  agrees within its accuracy.

FP32 and FP64 (the reference's DOUBLE_PRECISION) builds."""
import numpy as np
import pytest

import port
import tree_update as TU
from pipeline import assert_struct_equal
from tandav_b200 import gravity as G
from tandav_b200 import ics

pytestmark = pytest.mark.gpu

TREE_FIELDS = ("DNext", "Bitfield", "DUp", "Npart", "Pos", "Mass", "CoM", "Dp")
TOP_FIELDS = ("Key", "Target", "Level", "First_Part", "Npart", "Pos", "Mass", "CoM", "Dp")
DOMAIN_UPDATE_PARAM = 0.1           # the reference's Config value


def _case(kind):
    """Particles, domain and a Newtonian timeline whose time bins spread over
    six to eight rungs (chosen from the oracle's accelerations)."""
    if kind == "hernquist":
        p = ics.hernquist(n=8192, seed=21)
        c = np.median(p.pos, axis=1)
        size = 2.001 * np.abs(p.pos - c[:, None]).max()
        origin, t_end, dt_max = c - 0.5 * size, 0.02, 2e-3
    else:                                   # clumps in a periodic box
        p = ics.random_box(8192, box=2000.0, seed=22, clumps=9)
        origin, size, t_end, dt_max = np.zeros(3), p.box, 30.5, 1.9
    tl = dict(comoving=0, time_begin=0.0, time_end=t_end, hubble_constant=0.1, omega_matter=0.3,
              omega_lambda=0.7, omega_rad=0.0, omega_0=1.0, omega_baryon=0.0, rho_crit0=1.0,
              time_int_accuracy=0.025, max_timestep=dt_max, displ_constraint=0.25)
    return p, origin, size, tl


def _expected_kick(ctx, fsize):
    """The kept tree after the coming kick, restated from the device state."""
    d = ctx.download(G.F_MASS | G.F_ACC | G.F_TIME_BIN | G.F_IT_KICK | G.F_TREE_PARENT)
    tree, top = ctx.download_tree()
    st = ctx.timeline()
    active = np.flatnonzero(d["time_bin"] <= st.max_active_bin)
    ft = port.ftype(fsize)
    dt = np.zeros(len(d["mass"]), ft)
    factors = {}
    for i in active:
        c = int(d["it_kick_pos"][i])
        nx = c + ((1 << int(d["time_bin"][i])) >> 1)
        if (c, nx) not in factors:
            factors[(c, nx)] = ctx.kick_drift_factors(c, nx)[0]
        dt[i] = ft(factors[(c, nx)])
    dp = TU.particle_dp(d["mass"], dt, d["acc"], fsize)
    return TU.kicks(tree, top, d["tree_parent"], active, dp, fsize)


def _assert_tree(ctx, expected, what):
    tree, top = ctx.download_tree()
    assert_struct_equal(tree, expected[0], TREE_FIELDS, f"tree {what}")
    assert_struct_equal(top, expected[1], TOP_FIELDS, f"top nodes {what}")


@pytest.mark.parametrize("kind,fsize,flags", [("hernquist", 4, 0), ("hernquist", 8, 0), ("clumps", 4, 0),
                                              ("hernquist", 4, G.CFG_QUADRUPOLE)])
def test_tree_updates_in_the_step_loop(kind, fsize, flags):
    # (flags: with TVG_CFG_QUADRUPOLE the group form's node quadrupoles are
    # summed again from the drifted particles of the kept tree; the plain
    # form is unaffected)
    p, origin, size, timeline = _case(kind)
    ft = port.ftype(fsize)
    n = p.n
    prm = port.WalkParams(gravity=ics.GRAVITY, softening=p.softening, domain_size=size, boxsize=p.box,
                          open_bh=0.25, open_rel=0.005, use_bh=0, vector_size=64)
    group_check = fsize == 4 and p.box == 0
    seen = dict(kick=0, drift=0, walk=0, group=0)
    with G.GravityContext(n, float_bytes=fsize, periodic=p.box > 0, boxsize=p.box,
                          softening=p.softening, flags=flags) as ctx:
        ctx.upload(p.pos, p.mass, vel=p.vel, types=np.ones(n, np.int32),
                   time_bin=np.zeros(n, np.int32), it_drift=np.zeros(n, np.uint32),
                   it_kick=np.zeros(n, np.uint32))
        ctx.set_domain(origin, size)
        ctx.timeline_init(**timeline)
        # Update(BEFORE_MAIN_LOOP), update.c:13-34
        ctx.compute_acceleration(form=G.FORM_PLAIN, parts=G.WALK_GRAVITY, prepare=True)
        dom = ctx.time_for_domain_update(DOMAIN_UPDATE_PARAM)
        assert dom                                    # every particle was active
        for _ in range(16):
            ctx.set_new_timesteps()
            st = ctx.timeline()
            exp = None if dom else _expected_kick(ctx, fsize)
            ctx.kick_first_halfstep()
            if exp is not None:
                _assert_tree(ctx, exp, "after the first kick")
                seen["kick"] += 1
            drifted = not dom
            if drifted:
                tree, top = ctx.download_tree()
                exp = TU.drift(tree, top, st.time_step, fsize)
            ctx.drift_to_sync_point()
            if drifted:
                _assert_tree(ctx, exp, "after the drift")
                seen["drift"] += 1
            ids = ctx.download(G.F_ID)["id"]
            dom = ctx.time_for_domain_update(DOMAIN_UPDATE_PARAM)
            ctx.compute_acceleration(form=G.FORM_PLAIN, parts=G.WALK_GRAVITY)
            if not dom:
                d = ctx.download(G.F_ID | G.F_POS | G.F_MASS | G.F_GRAV_ACC | G.F_LAST_ACC
                                 | G.F_TIME_BIN)
                assert np.array_equal(d["id"], ids)   # no sort without a domain update
                tree, top = ctx.download_tree()
                act = d["time_bin"] <= ctx.timeline().max_active_bin
                g, _ = port.walk("gravity", d["pos"], d["mass"], d["last_acc_mag"], top, tree, prm,
                                 fsize=fsize)
                want, got = g.astype(ft)[:, act], d["grav_acc"][:, act]
                assert np.array_equal(got, want), f"walk on the kept tree: max diff " \
                                                  f"{np.abs(got.astype(float) - want).max()}"
                if drifted:
                    seen["walk"] += 1
                    if group_check and not seen["group"]:
                        # the group form on the same tree (it assigns Grav_Acc)
                        ctx.walk(G.FORM_GROUP, use_bh=False, parts=G.WALK_GRAVITY)
                        grp = ctx.download(G.F_GRAV_ACC)["grav_acc"][:, act].astype(np.float64)
                        ref = got.astype(np.float64)
                        err = np.sqrt(((grp - ref) ** 2).sum(0).mean() / (ref ** 2).sum(0).mean())
                        assert err < 1e-2, f"group form on the kept tree: rms {err:.2e}"
                        seen["group"] += 1
            exp = None if dom else _expected_kick(ctx, fsize)
            ctx.kick_second_halfstep()
            if exp is not None:
                _assert_tree(ctx, exp, "after the second kick")
                seen["kick"] += 1
    print(seen)
    assert seen["kick"] >= 6 and seen["drift"] >= 3 and seen["walk"] >= 2
    assert seen["group"] == (1 if group_check else 0)


@pytest.mark.parametrize("fsize", [4, 8])
def test_tree_kick_of_every_particle(fsize):
    """The first kick at a sync point that follows kept-tree steps adds every
    particle's momentum to the kept tree (the reference decides on the domain
    update only after that kick, main.c:49-67). There the top nodes and every
    node with more than 128 active particles are summed by a warp each; the
    tree must still equal the restatement bit for bit. A domain update
    parameter too large to trigger keeps the tree until the sync point."""
    p, origin, size, timeline = _case("hernquist")
    n = p.n
    with G.GravityContext(n, float_bytes=fsize, periodic=False, softening=p.softening) as ctx:
        ctx.upload(p.pos, p.mass, vel=p.vel, types=np.ones(n, np.int32),
                   time_bin=np.zeros(n, np.int32), it_drift=np.zeros(n, np.uint32),
                   it_kick=np.zeros(n, np.uint32))
        ctx.set_domain(origin, size)
        ctx.timeline_init(**timeline)
        ctx.compute_acceleration(form=G.FORM_PLAIN, parts=G.WALK_GRAVITY, prepare=True)
        dom = ctx.time_for_domain_update(1e6)
        kept = 0
        for _ in range(600):
            ctx.set_new_timesteps()
            st = ctx.timeline()
            if st.current >= st.end:
                break
            if not dom and st.n_active == n:
                exp = _expected_kick(ctx, fsize)
                ctx.kick_first_halfstep()
                _assert_tree(ctx, exp, "after a kick of every particle")
                return
            ctx.kick_first_halfstep()
            ctx.drift_to_sync_point()
            dom = ctx.time_for_domain_update(1e6)
            kept += int(not dom)
            ctx.compute_acceleration(form=G.FORM_PLAIN, parts=G.WALK_GRAVITY)
            ctx.kick_second_halfstep()
    pytest.fail(f"no sync point after {kept} kept-tree steps")
