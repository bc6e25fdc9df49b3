"""tvg_forcetest -- the GPU counterpart of Gravity_Forcetest
(src/Gravity/forcetest.c:25-172): FP64 direct summation with the reference's
softened kernel, Ewald-summed in a periodic box.

Pins: (1) at the nodes of the reference's Ewald table (Gravity/periodic.c:
368-411, computed in FP64 by the oracle with its own alpha = 2 sums) the
direct sum of one massive source must reproduce Newton + table value to FP64
round-off, since no interpolation is involved there; (2) on a Zel'dovich box
it must agree with the oracle's direct sum, which adds the tricubic
interpolant of that table per pair; (3) isolated, it must agree with the
oracle's plain direct sum; (4) the error statistics are those of the returned
arrays."""
import numpy as np
import pytest

import port
from tandav_b200 import gravity as G
from tandav_b200 import ics

pytestmark = pytest.mark.gpu


def sorted_targets(ctx, p, fsize, periodic, origin, size, ntgt, seed):
    ctx.upload(p.pos, p.mass)
    ctx.set_domain(origin, size)
    ctx.peano_keys()
    perm = ctx.sort_particles()
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(perm))
    tgt = np.random.default_rng(seed).choice(p.n, ntgt, replace=False)
    return tgt, inv[tgt].astype(np.int64)


def test_forcetest_table_nodes():
    L = 1000.0
    fx, fy, fz, _ = port.ewald_table(64)
    rng = np.random.default_rng(11)
    nodes = rng.integers(1, 64, size=(400, 3))
    x = nodes * (0.5 / 64)                               # box units, octant
    src = np.array([0.11, 0.17, 0.23]) * L
    pos = np.concatenate([src[:, None], src[:, None] + x.T * L], axis=1)
    m_src = 2.5e-3
    mass = np.zeros(pos.shape[1])
    mass[0] = m_src
    Gc = ics.GRAVITY
    with G.GravityContext(1024, float_bytes=8, periodic=True, boxsize=L, softening=1e-6) as ctx:
        ctx.upload(pos, mass)
        ad, _, _ = ctx.forcetest(np.arange(1, pos.shape[1]))
    d = -x * L                                          # source minus target
    r = np.sqrt((d ** 2).sum(1))
    newton = Gc * m_src * d / r[:, None] ** 3
    idx = (nodes[:, 0] * 65 + nodes[:, 1]) * 65 + nodes[:, 2]
    corr = np.stack([fx[idx], fy[idx], fz[idx]], axis=1) * Gc * m_src / L ** 2
    expect = (newton + corr).T
    scale = Gc * m_src / L ** 2
    err = np.abs(ad - expect).max() / scale
    print(f"max |a - (Newton + table)| = {err:.2e} G m / L^2")
    assert err < 1e-9


@pytest.mark.parametrize("fsize", [4, 8])
def test_forcetest_vs_oracle_periodic(fsize):
    p = ics.zeldovich_box(n_side=32, seed=32)
    ft = np.float32 if fsize == 4 else np.float64
    pos = p.pos.astype(ft).astype(np.float64)
    mass = p.mass.astype(ft).astype(np.float64)
    with G.GravityContext(p.n, float_bytes=fsize, periodic=True, boxsize=p.box,
                          softening=p.softening) as ctx:
        tgt, tsorted = sorted_targets(ctx, p, fsize, True, np.zeros(3), p.box, 400, 3)
        ad, _, _ = ctx.forcetest(tsorted)
        an, _, _ = ctx.forcetest(tsorted, parts=G.WALK_GRAVITY)
    # nearest image only: the plain FP64 sum
    ref_n = port.direct(pos, mass, tgt, ics.GRAVITY, p.softening, box=p.box)
    rel_n = np.sqrt(((an - ref_n) ** 2).sum(0) / (ref_n ** 2).sum(0))
    assert rel_n.max() < 1e-11
    fxt, fyt, fzt, _ = port.ewald_table(64)
    corr = np.stack([fxt, fyt, fzt], axis=1).reshape(-1).copy()
    ref = port.direct(pos, mass, tgt, ics.GRAVITY, p.softening, box=p.box, corr_table=corr,
                      corr_n=64)
    rel = np.sqrt(((ad - ref) ** 2).sum(0) / (ref ** 2).sum(0))
    print(f"Ewald sum vs tricubic table: rms {np.sqrt((rel ** 2).mean()):.2e} max {rel.max():.2e}")
    assert np.sqrt((rel ** 2).mean()) < 1e-5
    assert rel.max() < 1e-4


def test_forcetest_vs_oracle_isolated():
    p = ics.hernquist(n=20000, seed=7)
    c = np.median(p.pos, axis=1)
    size = 2.001 * np.abs(p.pos - c[:, None]).max()
    with G.GravityContext(p.n, float_bytes=8, periodic=False, softening=p.softening) as ctx:
        tgt, tsorted = sorted_targets(ctx, p, 8, False, c - 0.5 * size, size, 300, 4)
        ad, _, _ = ctx.forcetest(tsorted)
    ref = port.direct(p.pos, p.mass, tgt, ics.GRAVITY, p.softening)
    rel = np.sqrt(((ad - ref) ** 2).sum(0) / (ref ** 2).sum(0))
    print(f"isolated: max rel {rel.max():.2e}")
    assert rel.max() < 1e-12


def test_forcetest_error_statistics():
    p = ics.zeldovich_box(n_side=16, seed=5)
    with G.GravityContext(p.n, float_bytes=4, periodic=True, boxsize=p.box,
                          softening=p.softening) as ctx:
        ctx.upload(p.pos, p.mass)
        ctx.set_domain(np.zeros(3), p.box)
        ctx.ewald_init()
        ctx.force_step(form=G.FORM_GROUP, use_bh=True, parts=G.WALK_GRAVITY | G.WALK_EWALD)
        tgt = np.sort(np.random.default_rng(2).choice(p.n, 700, replace=False))
        ad, at, err = ctx.forcetest(tgt)
        ga = ctx.download(G.F_GRAV_ACC)["grav_acc"]
        with pytest.raises(G.TvgError):
            ctx.forcetest(np.array([p.n], np.int64))
        with pytest.raises(G.TvgError):
            ctx.forcetest(np.array([], np.int64))
    np.testing.assert_array_equal(at, ga[:, tgt].astype(np.float64))
    e = np.sqrt(((at - ad) ** 2).sum(0) / (ad ** 2).sum(0))
    es = np.sort(e)
    assert err["rms"] == pytest.approx(np.sqrt((e ** 2).mean()), rel=1e-12)
    assert err["p99"] == es[int(np.ceil(0.99 * len(e))) - 1]
    assert err["mean"] == pytest.approx(e.mean(), rel=1e-12)
    assert err["max"] == es[-1]
    assert err["rms"] < 5e-2
