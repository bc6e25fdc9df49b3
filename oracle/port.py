"""ctypes bindings of the oracle's C restatement (oracle/_ref/libtv_oracle.so).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path. Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg may import it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from refrun import TREE_DTYPE, TOPNODE_DTYPE

LIB_PATH = Path(__file__).resolve().parent / "_ref" / "libtv_oracle.so"
_lib = None


class WalkParams(C.Structure):
    _fields_ = [("gravity", C.c_double), ("softening", C.c_double),
                ("domain_size", C.c_double), ("boxsize", C.c_double),
                ("open_bh", C.c_double), ("open_rel", C.c_double),
                ("use_bh", C.c_int32), ("vector_size", C.c_int32)]


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} missing: run `make -C oracle port`")
        _lib = C.CDLL(str(LIB_PATH))
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def ftype(fsize):
    return np.float32 if fsize == 4 else np.float64


def peano_keys(pos, origin, size, fsize=4):
    """Std and reversed 128-bit keys as (n, 2) uint64 [hi, lo] arrays."""
    ft = ftype(fsize)
    x, y, z = (np.ascontiguousarray(pos[k], dtype=ft) for k in range(3))
    n = x.shape[0]
    std = np.zeros((n, 2), np.uint64)
    rev = np.zeros((n, 2), np.uint64)
    org = np.ascontiguousarray(origin, dtype=np.float64)
    lib().tvo_peano_keys(C.c_int64(n), C.c_int32(fsize), _p(x), _p(y), _p(z), _p(org),
                         C.c_double(size), _p(std), _p(rev))
    return std, rev


def sort_keys(keys):
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    n = keys.shape[0]
    perm = np.zeros(n, np.uint32)
    lib().tvo_sort_keys(C.c_int64(n), _p(keys), _p(perm))
    return perm


def top_nodes(std_sorted, pos_sorted, origin, size, fsize=4):
    ft = ftype(fsize)
    x, y, z = (np.ascontiguousarray(pos_sorted[k], dtype=ft) for k in range(3))
    out = np.zeros(64, TOPNODE_DTYPE)
    org = np.ascontiguousarray(origin, dtype=np.float64)
    k = np.ascontiguousarray(std_sorted, dtype=np.uint64)
    nt = lib().tvo_top_nodes(C.c_int64(x.shape[0]), C.c_int32(fsize), _p(k), _p(x), _p(y),
                             _p(z), _p(org), C.c_double(size), _p(out))
    return out[:nt].copy()


def tree_build(rev_sorted, pos_sorted, mass_sorted, domain_size, top, fsize=4, vector_size=64):
    """Returns (tree, top (updated), tree_parent). vector_size: the reference's
    compile-time VECTOR_SIZE (bundle size), 64 by default."""
    ft = ftype(fsize)
    x, y, z = (np.ascontiguousarray(pos_sorted[k], dtype=ft) for k in range(3))
    m = np.ascontiguousarray(mass_sorted, dtype=ft)
    n = x.shape[0]
    top = top.copy()
    cap = 2 * n + 1024
    tree = np.zeros(cap, TREE_DTYPE[fsize])
    parent = np.zeros(n, np.int32)
    rk = np.ascontiguousarray(rev_sorted, dtype=np.uint64)
    lib().tvo_tree_build.restype = C.c_int64
    nn = lib().tvo_tree_build(C.c_int64(n), C.c_int32(fsize), _p(rk), _p(x), _p(y), _p(z),
                              _p(m), C.c_double(domain_size), _p(top), C.c_int32(len(top)),
                              _p(tree), C.c_int64(cap), _p(parent), C.c_int32(vector_size))
    if nn < 0:
        raise RuntimeError(f"tvo_tree_build failed: {nn}")
    return tree[:nn].copy(), top, parent


def walk(kind, pos_sorted, mass_sorted, last_acc, top, tree, params: WalkParams,
         ewald_tables=None, fsize=4, potential=False):
    """kind = 'gravity' | 'ewald'; returns (acc (3, n) float64, cost (n,)),
    and with potential=True also the double sum of the potential terms (for
    'ewald' the fourth table of ewald_tables is the potential table)."""
    ft = ftype(fsize)
    x, y, z = (np.ascontiguousarray(pos_sorted[k], dtype=ft) for k in range(3))
    m = np.ascontiguousarray(mass_sorted, dtype=ft)
    la = np.ascontiguousarray(last_acc, dtype=ft)
    n = x.shape[0]
    acc = np.zeros((3, n))
    cost = np.zeros(n)
    top = np.ascontiguousarray(top)
    tree = np.ascontiguousarray(tree)
    pot = np.zeros(n) if potential else None
    if kind == "gravity":
        lib().tvo_walk_gravity_pot(C.c_int64(n), C.c_int32(fsize), _p(x), _p(y), _p(z), _p(m),
                                   _p(la), _p(top), C.c_int32(len(top)), _p(tree),
                                   C.byref(params), _p(acc), _p(cost), _p(pot))
    else:
        tabs = [np.ascontiguousarray(t, dtype=ft) for t in ewald_tables]
        fp = tabs[3] if potential else None
        lib().tvo_walk_ewald_pot(C.c_int64(n), C.c_int32(fsize), _p(x), _p(y), _p(z), _p(m),
                                 _p(la), _p(top), C.c_int32(len(top)), _p(tree),
                                 C.byref(params), _p(tabs[0]), _p(tabs[1]), _p(tabs[2]), _p(fp),
                                 _p(acc), _p(cost), _p(pot))
    return (acc, cost, pot) if potential else (acc, cost)


def ewald_table(n_ewald=64, potential=False):
    m = n_ewald + 1
    fx, fy, fz = (np.zeros(m ** 3) for _ in range(3))
    fp = np.zeros(m ** 3) if potential else None
    lib().tvo_ewald_table(C.c_int32(n_ewald), _p(fx), _p(fy), _p(fz), _p(fp))
    return fx, fy, fz, fp


def ewald_force(x, nreal=4, nk=4):
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
    f = np.zeros_like(x)
    lib().tvo_ewald_force(C.c_int64(x.shape[0]), _p(x), C.c_int32(nreal), C.c_int32(nk), _p(f))
    return f


def direct(pos, mass, targets, gravity, softening, box=0.0, corr_table=None, corr_n=0):
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    t = np.ascontiguousarray(targets, dtype=np.int64)
    acc = np.zeros((3, t.shape[0]))
    ct = None if corr_table is None else np.ascontiguousarray(corr_table, dtype=np.float64)
    lib().tvo_direct(C.c_int64(mass.shape[0]), _p(pos), _p(mass), C.c_int64(t.shape[0]), _p(t),
                     C.c_double(gravity), C.c_double(softening), C.c_double(box), _p(ct),
                     C.c_int32(corr_n), _p(acc))
    return acc


def find_domain(pos, fsize=4, box=0.0):
    """set_computational_domain (src/domain.c:732-847) restated: periodic ->
    (origin 0, size box); isolated -> centre = Median of each coordinate as
    select.c computes it, Select(n >> 1, n, data) with the 1-based Numerical
    Recipes bounds on a 0-based array, i.e. the (n >> 1)-th smallest of
    data[1 .. n-1] (data[0] for n = 1), kept in Float; size = 2.001 * the
    largest |x - centre| (double); origin = centre - size / 2."""
    if box > 0:
        return np.zeros(3), float(box)
    p = np.asarray(pos, dtype=ftype(fsize))
    n = p.shape[1]
    center = np.zeros(3)
    for d in range(3):
        if n == 1:
            center[d] = float(p[d, 0])
        else:
            k = n >> 1
            center[d] = float(np.partition(p[d, 1:], k - 1)[k - 1])
    maxd = float(np.abs(p.astype(np.float64) - center[:, None]).max())
    size = 2.001 * maxd
    return center - 0.5 * size, size
