"""Host memory registered with tvg_host_register, as the reference's single
memory pool holding P would be: uploads from and downloads into arrays
carved out of one registered pool carry the data unchanged; a second
registration of the pool and the release of an unregistered range are
TVG_E_STATE."""
import ctypes as C

import numpy as np
import pytest

from tandav_b200 import gravity as G
from tandav_b200 import ics

pytestmark = pytest.mark.gpu


def test_registered_pool_round_trip():
    p = ics.zeldovich_box(n_side=16, seed=3)
    n = p.n
    pool = np.zeros(7 * n * 4, np.uint8)                 # pos, mass, out: float32
    pos = pool[: 3 * n * 4].view(np.float32).reshape(3, n)
    mass = pool[3 * n * 4: 4 * n * 4].view(np.float32)
    out = pool[4 * n * 4:].view(np.float32).reshape(3, n)
    pos[:] = p.pos
    mass[:] = p.mass
    lib = G.lib()
    G.host_register(pool)
    try:
        assert lib.tvg_host_register(C.c_void_p(pool.ctypes.data), C.c_size_t(pool.nbytes)) == 7
        with G.GravityContext(n, float_bytes=4, periodic=True, boxsize=p.box,
                              softening=p.softening) as ctx:
            ctx.upload(pos, mass)                        # rows of the pool, no copies
            q = G.Particles()
            for k in range(3):
                q.pos[k] = out[k].ctypes.data
            assert lib.tvg_download(ctx.ctx, C.byref(q), C.c_uint32(G.F_POS)) == G.TVG_OK
        np.testing.assert_array_equal(out, pos)
    finally:
        G.host_unregister(pool)
    assert lib.tvg_host_unregister(C.c_void_p(pool.ctypes.data)) == 7
