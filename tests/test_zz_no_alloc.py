"""The sort entry point that allocates nothing (tvg_sort_keys_noalloc).

It exists for callers that cannot allocate device memory -- a host code whose
own memory manager reserves the GPU's memory up front and admits no other
allocation, or a step loop that cannot take the device-wide synchronisation
of cudaMalloc and cudaFree -- and keeps its scratch in a fixed device array
instead. Here the caller's device buffers are torch tensors; the permutation
must equal the one the context-based sort (tvg_sort_particles) returns for
the same keys, bit for bit, on two calls in a row (the second on different,
smaller input, so stale scratch from the first call would show), and a call
must leave the device's free memory unchanged.
"""
import ctypes as C

import numpy as np
import pytest

import tandav_b200
from tandav_b200 import gravity as G
from tandav_b200 import ics

pytestmark = pytest.mark.gpu

MAX_KEYS = 1 << 18        # TVG_NOALLOC_MAX_KEYS in include/tandav_gpu.h


def context_keys_and_perm(p):
    """Keys (input order) and the permutation of the existing entry point."""
    with G.GravityContext(p.n, float_bytes=4, periodic=True, boxsize=p.box,
                          softening=p.softening) as ctx:
        ctx.upload(p.pos, p.mass)
        ctx.set_domain((0.0, 0.0, 0.0), p.box)
        ctx.peano_keys()
        keys = ctx.download(G.F_KEY)["key"]          # (n, 2) [hi, lo]
        perm = ctx.sort_particles()
    return keys, perm


def noalloc_perm(keys):
    """Permutation from tvg_sort_keys_noalloc, and the device's free memory
    just before and just after the call (all buffers made beforehand)."""
    import torch
    n = keys.shape[0]
    hi = torch.from_numpy(np.ascontiguousarray(keys[:, 0]).view(np.int64)).cuda()
    lo = torch.from_numpy(np.ascontiguousarray(keys[:, 1]).view(np.int64)).cuda()
    out = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    rc = tandav_b200.lib().tvg_sort_keys_noalloc(C.c_void_p(hi.data_ptr()), C.c_void_p(lo.data_ptr()),
                                                 C.c_int64(n), C.c_void_p(out.data_ptr()))
    free_after = torch.cuda.mem_get_info()[0]
    assert rc == 0, f"tvg_sort_keys_noalloc returned {rc}"
    return out.cpu().numpy().view(np.uint32), free_before, free_after


def test_noalloc_sort_matches_context_sort_twice():
    first = ics.random_box(200000, box=1000.0, seed=41, clumps=7)
    second = ics.random_box(150001, box=1000.0, seed=42, clumps=3)
    # coincident particles: equal 128-bit keys keep input order in both paths
    second.pos[:, 100:110] = second.pos[:, 5:6]
    for k, p in enumerate((first, second)):
        keys, perm_ref = context_keys_and_perm(p)
        perm, free_before, free_after = noalloc_perm(keys)
        assert np.array_equal(perm, perm_ref)
        if k > 0:     # the first call may load the module; later calls allocate nothing
            assert free_after == free_before, (free_before, free_after)


def test_noalloc_rejects_oversized_input():
    import torch
    buf = torch.zeros(4, dtype=torch.int64, device="cuda")
    rc = tandav_b200.lib().tvg_sort_keys_noalloc(C.c_void_p(buf.data_ptr()), C.c_void_p(buf.data_ptr()),
                                                 C.c_int64(MAX_KEYS + 1), C.c_void_p(buf.data_ptr()))
    assert rc == 5                                    # TVG_E_BADINPUT


def test_noalloc_sort_orders_long_runs_of_equal_high_words():
    """Keys whose high words repeat in runs of thousands (particles packed in
    one cell of the 21st level share them): each run comes out ordered by the
    low word and stable for equal keys, as numpy's lexicographic sort gives."""
    rng = np.random.default_rng(43)
    n = 200000
    hi = rng.integers(0, 2 ** 63, size=n, dtype=np.uint64)
    runs = rng.choice(n, 30000, replace=False)
    hi[runs] = rng.choice(np.array([3, 17, 2 ** 40 + 5, 2 ** 62 + 1], dtype=np.uint64), size=len(runs),
                          p=[0.5, 0.3, 0.15, 0.05])
    lo = rng.integers(0, 2 ** 20, size=n, dtype=np.uint64)   # with repeats
    keys = np.stack([hi, lo], axis=1)
    perm, _, _ = noalloc_perm(keys)
    assert np.array_equal(perm, np.lexsort((lo, hi)).astype(np.uint32))
