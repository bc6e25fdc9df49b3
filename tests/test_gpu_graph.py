"""The step as one CUDA graph (tvg_step_graph, tvg_step.cu): launches of the
captured Compute_Acceleration give bit for bit the accelerations, particle
order, tree and counts of the step run directly, for all particles and for
the active particles of a hierarchical step loop (src/main.c:43-70), where
each graph launch reads the current active-bin limit and active count on the
device."""
import numpy as np
import pytest

from tandav_b200 import gravity as G
from tandav_b200 import ics

pytestmark = pytest.mark.gpu

PARTS = G.WALK_GRAVITY | G.WALK_EWALD
FIELDS = G.F_ACC | G.F_GRAV_ACC | G.F_ID | G.F_POS | G.F_VEL | G.F_LAST_ACC


def _ctx(p, flags=0):
    ctx = G.GravityContext(p.n, float_bytes=4, periodic=True, boxsize=p.box, softening=p.softening,
                           flags=flags)
    ctx.set_domain((0, 0, 0), p.box)
    ctx.ewald_init()
    ctx.set_opening(0.25, 2e-4)
    return ctx


def _same(a, b):
    for k in a:
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)


@pytest.mark.parametrize("flags", [0, G.CFG_QUADRUPOLE])
def test_graph_step_equals_direct_step(flags):
    p = ics.zeldovich_box(n_side=32, seed=41)
    direct, graph = _ctx(p, flags), _ctx(p, flags)
    try:
        for c in (direct, graph):
            c.upload(p.pos, p.mass)
            c.compute_acceleration(form=G.FORM_GROUP, parts=PARTS, prepare=True)
        l0 = graph.launch_count()
        for _ in range(5):
            direct.compute_acceleration(form=G.FORM_GROUP, parts=PARTS)
            graph.step_graph(PARTS)
            _same(direct.download(FIELDS), graph.download(FIELDS))
            assert direct.walk_counters() == graph.walk_counters()
            assert direct.walk_quad_interactions() == graph.walk_quad_interactions()
            assert (graph.walk_quad_interactions() > 0) == bool(flags)
            (tree_d, top_d), (tree_g, top_g) = direct.download_tree(), graph.download_tree()
            assert tree_d.tobytes() == tree_g.tobytes() and top_d.tobytes() == top_g.tobytes()
        # the captured steps' kernels are counted per launch
        assert graph.launch_count() > l0
    finally:
        direct.close()
        graph.close()


def _loop_ctx(p, flags=0):
    ctx = _ctx(p, flags)
    n = p.n
    ctx.upload(p.pos, p.mass, vel=p.vel, types=np.ones(n, np.int32), time_bin=np.zeros(n, np.int32),
               it_drift=np.zeros(n, np.uint32), it_kick=np.zeros(n, np.uint32))
    ctx.timeline_init(comoving=1, time_begin=p.a_start, time_end=1.0, hubble_constant=0.1,
                      omega_matter=0.3, omega_lambda=0.7, omega_rad=0.0, omega_0=1.0,
                      omega_baryon=0.0, rho_crit0=3 * 0.01 / (8 * np.pi * ics.GRAVITY),
                      time_int_accuracy=0.01, max_timestep=0.05, displ_constraint=0.25)
    ctx.compute_acceleration(form=G.FORM_GROUP, parts=PARTS, prepare=True)
    return ctx


@pytest.mark.parametrize("flags", [0, G.CFG_QUADRUPOLE])
def test_graph_step_in_the_step_loop(flags):
    p = ics.zeldovich_box(n_side=32, seed=42)
    direct, graph = _loop_ctx(p, flags), _loop_ctx(p, flags)
    try:
        actives = set()
        for _ in range(8):
            for c, use_graph in ((direct, False), (graph, True)):
                c.set_new_timesteps()
                c.kick_first_halfstep()
                c.drift_to_sync_point()
                if use_graph:
                    c.step_graph(PARTS)
                else:
                    c.compute_acceleration(form=G.FORM_GROUP, parts=PARTS)
                c.kick_second_halfstep()
            sd, sg = direct.timeline(), graph.timeline()
            assert (sd.current, sd.n_active, sd.max_active_bin) == (sg.current, sg.n_active,
                                                                    sg.max_active_bin)
            actives.add(sd.n_active)
            _same(direct.download(FIELDS), graph.download(FIELDS))
        # steps with different active sets went through the captured graphs
        assert len(actives) > 1
    finally:
        direct.close()
        graph.close()


def test_graph_follows_parameter_changes():
    # the opening parameters are passed to the captured kernels by value: a
    # change must give a new capture, not a replay with the old values
    p = ics.zeldovich_box(n_side=32, seed=43)
    direct, graph = _ctx(p), _ctx(p)
    try:
        for c in (direct, graph):
            c.upload(p.pos, p.mass)
            c.compute_acceleration(form=G.FORM_GROUP, parts=PARTS, prepare=True)
        for setting in (None, ("open", 0.25, 5e-4), ("ewald", 1e-3, 0.5), None):
            if setting and setting[0] == "open":
                for c in (direct, graph):
                    c.set_opening(setting[1], setting[2])
            elif setting:
                for c in (direct, graph):
                    c.set_ewald_opening(setting[1], setting[2])
            for _ in range(3):          # a direct step, then the two captures / replays
                direct.compute_acceleration(form=G.FORM_GROUP, parts=PARTS)
                graph.step_graph(PARTS)
                _same(direct.download(FIELDS), graph.download(FIELDS))
                assert direct.walk_counters() == graph.walk_counters()
    finally:
        direct.close()
        graph.close()
