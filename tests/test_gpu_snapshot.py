"""Snapshot of the resident particles (tvg_write_snapshot): after a force step
(keys, sort, build, walks on the device) the file holds the particles in
their Peano-Hilbert order with their IDs, Acc[0], Grav_Acc and (FP64 with
GRAVITY_POTENTIAL) Grav_Pot, and equals
byte for byte the file the host writer makes from the downloaded fields. The
host writer itself is pinned to the reference's Write_Snapshot in
test_snapshot.py."""
import numpy as np
import pytest

from tandav_b200 import gravity as G
from tandav_b200 import ics

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fb,potential", [(4, False), (8, True)])
def test_device_snapshot_equals_host_writer(tmp_path, fb, potential):
    p = ics.zeldovich_box(n_side=24, seed=17)
    ft = np.float32 if fb == 4 else np.float64
    ids = np.arange(p.n, dtype=np.uint32)
    flags = G.CFG_POTENTIAL if potential else 0
    with G.GravityContext(p.n, float_bytes=fb, periodic=True, boxsize=p.box,
                          softening=p.softening, flags=flags) as ctx:
        ctx.upload(p.pos, p.mass, vel=p.vel, ids=ids)
        ctx.set_domain((0, 0, 0), p.box)
        ctx.ewald_init()
        form = G.FORM_GROUP if fb == 4 else G.FORM_PLAIN
        ctx.force_step(form=form, use_bh=True, parts=G.WALK_GRAVITY | G.WALK_EWALD)
        h = G.snapshot_header(p.n, p.a_start, p.box, 0.3, 0.7, 0.7)
        blocks = G.SNAP_ACC | G.SNAP_GACC | (G.SNAP_GPOT if potential else 0)
        ctx.write_snapshot(tmp_path / "dev_000", h, blocks)
        d = ctx.download(G.F_POS | G.F_VEL | G.F_ID | G.F_MASS | G.F_ACC | G.F_GRAV_ACC
                         | (G.F_GRAV_POT if potential else 0))
    G.write_snapshot_host(tmp_path / "host_000", h, d["pos"], d["vel"], d["id"], d["mass"],
                          acc=d["acc"], grav_acc=d["grav_acc"], grav_pot=d.get("grav_pot"))
    assert (tmp_path / "dev_000").read_bytes() == (tmp_path / "host_000").read_bytes()
    # sorted order: the IDs are a permutation and carry their particles along
    assert np.array_equal(np.sort(d["id"]), ids)
    assert not np.array_equal(d["id"], ids)
    np.testing.assert_array_equal(d["pos"], p.pos.astype(ft)[:, d["id"]])
    np.testing.assert_array_equal(d["vel"], p.vel.astype(ft)[:, d["id"]])
    assert np.all(np.isfinite(d["grav_acc"])) and np.any(d["grav_acc"] != 0)
    if potential:
        assert np.all(np.isfinite(d["grav_pot"])) and np.any(d["grav_pot"] != 0)


def test_read_snapshot_to_device(tmp_path):
    """tvg_read_snapshot: a two-type snapshot read onto the device holds the
    particles the host reader returns, field for field and in its order."""
    rng = np.random.default_rng(8)
    n1, n4 = 3000, 1000
    n = n1 + n4
    pos = rng.uniform(0, 100.0, (3, n)).astype(np.float32)
    vel = rng.normal(0, 30.0, (3, n)).astype(np.float32)
    mass = rng.uniform(0.5, 1.5, n).astype(np.float32)
    gacc = rng.normal(0, 1.0, (3, n)).astype(np.float32)
    ids = np.concatenate([rng.permutation(n1), n1 + rng.permutation(n4)]).astype(np.uint32)
    h = G.snapshot_header([0, n1, 0, 0, n4, 0], 0.5, 100.0)
    path = tmp_path / "ics"
    G.write_snapshot_host(path, h, pos, vel, ids, mass, grav_acc=gacc)
    host = G.read_snapshot(path, 4)
    with G.GravityContext(n, float_bytes=4, periodic=True, boxsize=100.0, softening=0.1) as ctx:
        got_n, blocks = ctx.read_snapshot(path)
        d = ctx.download(G.F_POS | G.F_VEL | G.F_ID | G.F_MASS | G.F_TYPE | G.F_GRAV_ACC)
    assert got_n == n and blocks == G.SNAP_MASS | G.SNAP_GACC
    for k in ("pos", "vel", "id", "mass", "type", "grav_acc"):
        np.testing.assert_array_equal(d[k], host[k], err_msg=k)
    np.testing.assert_array_equal(np.unique(d["type"]), [1, 4])
