"""tvg_force_step_host against the three calls it overlaps (tvg_upload,
tvg_force_step, tvg_download) on the same pinned host buffers: the
accelerations and the particle IDs in the new PH order must be the same bit
for bit, for a Barnes-Hut step and a relative-criterion step that takes
|a_old| from it, twice in a row; in a periodic box with the Ewald walk and
node quadrupoles, and in isolation with the domain found at every step
(TVG_CFG_FIND_DOMAIN). Calls without positions are refused."""
import ctypes as C

import numpy as np
import pytest

from tandav_b200 import gravity as G
from tandav_b200 import ics

pytestmark = pytest.mark.gpu


def _pinned(shape, dtype):
    return G.PinnedArray(shape, dtype)


def _run_both(ctx, n, pos, mass, last, ids, use_bh, parts):
    acc_a = _pinned((3, n), np.float32)
    ids_a = _pinned((n,), np.uint32)
    ctx.upload_fields(n, pos=pos, mass=mass, last_acc=last, ids=ids)
    ctx.force_step(form=G.FORM_GROUP, use_bh=use_bh, parts=parts)
    ctx.download_into(grav_acc=acc_a.array, ids=ids_a.array)
    acc_b = _pinned((3, n), np.float32)
    ids_b = _pinned((n,), np.uint32)
    ctx.force_step_host(n, pos, mass, last_acc=last, ids=ids, grav_acc=acc_b.array, ids_out=ids_b.array,
                        form=G.FORM_GROUP, use_bh=use_bh, parts=parts)
    return (acc_a.array.copy(), ids_a.array.copy()), (acc_b.array.copy(), ids_b.array.copy())


@pytest.mark.parametrize("case", ["periodic_quadrupole", "isolated_find_domain"])
def test_force_step_host_equals_the_three_calls(case):
    if case == "periodic_quadrupole":
        p = ics.zeldovich_box(n_side=32, seed=17)
        kw = dict(periodic=True, boxsize=p.box, flags=G.CFG_QUADRUPOLE)
        parts = G.WALK_GRAVITY | G.WALK_EWALD
    else:
        p = ics.hernquist(n=20000, seed=5)
        kw = dict(periodic=False, boxsize=0.0, flags=G.CFG_FIND_DOMAIN)
        parts = G.WALK_GRAVITY
    n = p.n
    pos = _pinned((3, n), np.float32)
    mass = _pinned((n,), np.float32)
    last = _pinned((n,), np.float32)
    ids = _pinned((n,), np.uint32)
    pos.array[:] = p.pos.astype(np.float32)
    mass.array[:] = p.mass.astype(np.float32)
    ids.array[:] = np.arange(n, dtype=np.uint32)
    last.array[:] = 0.0
    with G.GravityContext(n, float_bytes=4, softening=p.softening, **kw) as ctx:
        if p.box > 0:
            ctx.set_domain((0.0, 0.0, 0.0), p.box)
        # Barnes-Hut, then the relative criterion with |a_old| from it, twice
        a, b = _run_both(ctx, n, pos.array, mass.array, last.array, ids.array, True, parts)
        assert np.array_equal(a[1], b[1])
        assert np.array_equal(a[0], b[0])
        last.array[b[1]] = np.sqrt((b[0].astype(np.float64) ** 2).sum(0)).astype(np.float32)
        for _ in range(2):
            a, b = _run_both(ctx, n, pos.array, mass.array, last.array, ids.array, False, parts)
            assert np.array_equal(a[1], b[1])
            assert np.array_equal(a[0], b[0])
            assert np.all(np.isfinite(b[0])) and np.abs(b[0]).max() > 0
        # the positions are a required input
        src, dst = G.Particles(), G.Particles()
        src.mass = mass.array.ctypes.data
        rc = G.lib().tvg_force_step_host(ctx.ctx, C.c_int64(n), C.byref(src), C.c_uint32(G.F_MASS),
                                         C.byref(dst), C.c_uint32(0), C.c_int32(G.FORM_GROUP), C.c_int32(0),
                                         C.c_uint32(parts), C.c_int32(G.EWALD_TABLE))
        assert rc == 5                                  # TVG_E_BADINPUT
