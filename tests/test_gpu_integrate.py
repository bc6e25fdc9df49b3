"""Hierarchical time integration on the GPU (tvg_integrate.cu) against the
oracle restatement of the reference (oracle/integrate.py): comoving kick and
drift tables (Einstein-de Sitter closed forms, adaptive quadrature for
LCDM), time bins, kick, drift and wrap bit for bit, the timeline logic, and a
short run of the full step loop (src/main.c:43-70) against linear growth."""
import math

import numpy as np
import pytest

import integrate as O
from tandav_b200 import gravity as G
from tandav_b200 import ics

pytestmark = pytest.mark.gpu

H0 = 0.1
RHO_CRIT0 = 3.0 * H0 ** 2 / (8.0 * math.pi * ics.GRAVITY)


def timeline_cfg(**kw):
    cfg = dict(comoving=1, time_begin=1.0 / 51.0, time_end=1.0, hubble_constant=H0,
               omega_matter=0.3, omega_lambda=0.7, omega_rad=0.0, omega_0=1.0, omega_baryon=0.0,
               rho_crit0=RHO_CRIT0, time_int_accuracy=0.025, max_timestep=0.05,
               displ_constraint=0.25)
    cfg.update(kw)
    return cfg


def test_kd_table_einstein_de_sitter():
    with G.GravityContext(1024, periodic=True, boxsize=1000.0) as ctx:
        ctx.timeline_init(**timeline_cfg(omega_matter=1.0, omega_lambda=0.0))
        a, k, d = ctx.kick_drift_table()
        x, a0, _ = O.knots(1.0 / 51.0, 1.0)
        np.testing.assert_allclose(a[1:], x[1:], rtol=1e-14)
        assert a[0] == 0 and k[0] == 0 and d[0] == 0
        kick = 2.0 / H0 * (np.sqrt(x[1:]) - math.sqrt(a0))
        drift = -2.0 / H0 * (1.0 / np.sqrt(x[1:]) - 1.0 / math.sqrt(a0))
        np.testing.assert_allclose(k[1:], kick, rtol=1e-12)
        np.testing.assert_allclose(d[1:], drift, rtol=1e-12)
        st = ctx.timeline()
        rng = np.random.default_rng(3)
        for _ in range(20):
            c = int(rng.integers(0, 1 << 30))
            n = c + int(rng.integers(1 << 20, 1 << 30))
            kf, df = ctx.kick_drift_factors(c, n)
            a_c = st.time_current * math.exp(c * st.step_min)
            a_n = st.time_current * math.exp(n * st.step_min)
            assert kf == pytest.approx(2.0 / H0 * (math.sqrt(a_n) - math.sqrt(a_c)), rel=1e-7)
            assert df == pytest.approx(-2.0 / H0 * (1 / math.sqrt(a_n) - 1 / math.sqrt(a_c)), rel=1e-7)


def test_kd_table_lcdm_vs_quadrature():
    with G.GravityContext(1024, periodic=True, boxsize=1000.0) as ctx:
        ctx.timeline_init(**timeline_cfg())
        a, k, d = ctx.kick_drift_table()
        st = ctx.timeline()
        cosmo = (H0, 0.3, 0.7, 0.0, 1.0)
        x, kq, dq = O.kd_integrals(1.0 / 51.0, 1.0, cosmo)
        np.testing.assert_allclose(k[1:], kq[1:], rtol=1e-10)
        np.testing.assert_allclose(d[1:], dq[1:], rtol=1e-10)
        # the spline through the oracle's table gives the same factors
        m2k, m2d = O.natural_spline(x, kq), O.natural_spline(x, dq)
        for c, n in ((0, 1 << 24), (1 << 20, (1 << 20) + (1 << 22)), (1 << 30, (1 << 31) - 1)):
            kf, df = ctx.kick_drift_factors(c, n)
            ac, an = st.time_current * math.exp(c * st.step_min), st.time_current * math.exp(n * st.step_min)
            ko = O.spline_eval(x, kq, m2k, an) - O.spline_eval(x, kq, m2k, ac)
            do = O.spline_eval(x, dq, m2d, an) - O.spline_eval(x, dq, m2d, ac)
            assert kf == pytest.approx(ko, rel=1e-9)
            assert df == pytest.approx(do, rel=1e-9)


@pytest.mark.parametrize("fsize", [4, 8])
def test_timebins_kick_drift_wrap_parity(fsize):
    p = ics.zeldovich_box(n_side=16, seed=4)
    n = p.n
    rng = np.random.default_rng(9)
    ft = np.float32 if fsize == 4 else np.float64
    gacc = (rng.standard_normal((3, n)) * 300.0).astype(ft)
    acc = (rng.standard_normal((3, n)) * 300.0).astype(ft)
    bins = rng.integers(0, 20, n).astype(np.int32)
    types = np.ones(n, np.int32)
    zeros = np.zeros(n, np.uint32)
    pos = p.pos.copy()
    pos[0, :5] = [-3.0, p.box + 2.0, -2.5 * p.box, 0.0, p.box]      # needs wrapping
    with G.GravityContext(n, float_bytes=fsize, periodic=True, boxsize=p.box,
                          softening=p.softening) as ctx:
        ctx.upload(pos, p.mass, vel=p.vel, types=types, time_bin=bins, it_drift=zeros,
                   it_kick=zeros, acc=acc, grav_acc=gacc)
        cfg = timeline_cfg()
        ctx.timeline_init(**cfg)
        st0 = ctx.timeline()
        ctx.set_new_timesteps()
        st = ctx.timeline()
        dev = ctx.download(G.F_TIME_BIN | G.F_VEL | G.F_POS)
        # Dt_Max_Global from the velocity dispersion (comoving.c:195-287)
        v = [np.asarray(p.vel[k], ft) for k in range(3)]
        vel2 = float(np.sum(((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]).astype(np.float64)))
        dmean = (float(np.float32(p.mass[0])) / (0.3 * RHO_CRIT0)) ** (1 / 3)
        dtv = 0.25 * dmean / math.sqrt(vel2 / n) * st0.expansion_factor ** 2 * st0.hubble_parameter
        assert st.dt_max_global == pytest.approx(np.float32(min(cfg["max_timestep"], dtv)), rel=1e-6)
        ob = O.timebins(gacc, np.zeros(n, np.int32) + bins, float_bytes=fsize, comoving=1,
                        expansion_factor=st0.expansion_factor, hubble_parameter=st0.hubble_parameter,
                        time_int_accuracy=cfg["time_int_accuracy"], softening=p.softening,
                        step_max=st0.step_max, dt_max_global=st.dt_max_global,
                        max_active_bin=st0.max_active_bin)
        np.testing.assert_array_equal(dev["time_bin"], ob)
        assert (st.time_bin_min, st.time_bin_max) == (ob.min(), ob.max())
        so = O.system_step(dict(beg=st0.beg, current=st0.current, end=st0.end,
                                next_sync_point=st0.next_sync_point, time_current=st0.time_current),
                           int(ob.min()), int(ob.max()),
                           lambda it: st0.time_current * math.exp(it * st0.step_min))
        for key in ("step", "next", "max_active_bin", "sync_point", "next_sync_point"):
            assert getattr(st, key) == so[key], key
        active = np.nonzero(ob <= so["max_active_bin"])[0]
        assert st.n_active == len(active)
        # kick (all the arithmetic of kick.c, factors from the device spline)
        ctx.kick_first_halfstep()
        dev2 = ctx.download(G.F_VEL | G.F_IT_KICK)
        vo, itk = O.kick(p.vel, acc, ob, zeros, active,
                         lambda c, nx: ctx.kick_drift_factors(c, nx)[0], fsize)
        for k in range(3):
            np.testing.assert_array_equal(dev2["vel"][k], vo[k])
        np.testing.assert_array_equal(dev2["it_kick_pos"], itk)
        # drift + wrap + clock
        ctx.drift_to_sync_point()
        st2 = ctx.timeline()
        dev3 = ctx.download(G.F_POS | G.F_IT_DRIFT)
        xo, itd = O.drift(pos, vo, zeros, active, st.next,
                          lambda c, nx: ctx.kick_drift_factors(c, nx)[1], fsize)
        xo = O.wrap(xo, p.box, fsize)
        for k in range(3):
            np.testing.assert_array_equal(dev3["pos"][k], xo[k])
        np.testing.assert_array_equal(dev3["it_drift_pos"], itd)
        assert st2.current == st.current + st.step and st2.step_counter == 1
        assert st2.time_current == pytest.approx(st.time_next, rel=1e-15)


def test_rung_run_linear_growth():
    """The step loop of src/main.c:43-70 on a 32^3 box from z = 50 to z ~ 35;
    the displacement field must grow like the linear growth factor."""
    cosmo = ics.Cosmology()
    p = ics.zeldovich_box(n_side=32, seed=21, z_start=50.0)
    n, L = p.n, p.box
    spacing = L / 32
    g = (np.arange(32) + 0.5) * spacing
    q = np.stack(np.meshgrid(g, g, g, indexing="ij")).reshape(3, -1)

    def disp(pos):
        d = pos - q
        return d - L * np.round(d / L)

    a_end = 1.0 / 36.0
    with G.GravityContext(n, float_bytes=4, periodic=True, boxsize=L, softening=p.softening) as ctx:
        ctx.upload(p.pos, p.mass, vel=p.vel, types=np.ones(n, np.int32),
                   time_bin=np.zeros(n, np.int32), it_drift=np.zeros(n, np.uint32),
                   it_kick=np.zeros(n, np.uint32))
        ctx.set_domain((0, 0, 0), L)
        ctx.ewald_init()
        ctx.timeline_init(**timeline_cfg(time_begin=p.a_start, time_end=a_end,
                                         time_int_accuracy=0.02))
        parts = G.WALK_GRAVITY | G.WALK_EWALD
        ctx.compute_acceleration(form=G.FORM_GROUP, parts=parts, prepare=True)
        hist_used = np.zeros(32, np.int64)
        steps = 0
        while True:
            st = ctx.timeline()
            if st.current >= st.end:
                break
            ctx.set_new_timesteps()
            st = ctx.timeline()
            h = ctx.rung_histogram()
            hist_used += h > 0
            assert st.n_active == int(h[: st.max_active_bin + 1].sum())
            ctx.kick_first_halfstep()
            ctx.drift_to_sync_point()
            ctx.compute_acceleration(form=G.FORM_GROUP, parts=parts)
            ctx.kick_second_halfstep()
            steps += 1
            assert steps < 5000
        out = ctx.download(G.F_POS | G.F_ID | G.F_IT_KICK | G.F_IT_DRIFT)
        st = ctx.timeline()
    assert st.current == st.end
    np.testing.assert_array_equal(out["it_kick_pos"], out["it_drift_pos"])
    inv = np.argsort(out["id"])
    d0 = disp(p.pos)
    d1 = disp(out["pos"][:, inv].astype(np.float64))
    growth = cosmo.growth(a_end) / cosmo.growth(p.a_start)
    pred = d0 * growth
    rel = np.sqrt(((d1 - pred) ** 2).sum() / ((pred - d0) ** 2).sum())
    print(f"steps {steps}, rungs used {int((hist_used > 0).sum())}, growth {growth:.4f}, "
          f"|d1 - D d0| / |(D - 1) d0| = {rel:.3e}")
    assert (hist_used > 0).sum() >= 2
    assert rel < 0.05
