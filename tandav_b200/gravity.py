"""Python view of the C ABI (include/tandav_gpu.h), one method per entry point.

The method names follow the reference entry points they replace
(src/peano.c, src/Gravity/tree_build.c, tree_accel.c, tree_periodic.c,
Gravity/periodic.c, kick.c, drift.c). Arrays are numpy; the Float width is
``float_bytes`` (4 or 8, the reference's DOUBLE_PRECISION switch).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import lib
from .ics import GRAVITY

TVG_OK = 0
ERRORS = {1: "TVG_E_CUDA", 2: "TVG_E_NOMEM", 3: "TVG_E_TREE_FULL", 4: "TVG_E_TIMEOUT",
          5: "TVG_E_BADINPUT", 6: "TVG_E_COINCIDENT", 7: "TVG_E_STATE"}

FORM_PLAIN, FORM_GROUP = 0, 1
WALK_GRAVITY, WALK_EWALD = 1, 2
EWALD_TABLE, EWALD_MLP = 0, 1
BUILD_EXACT_MOMENTS = 1
CFG_FIX_SMALL_TOPNODES = 1
CFG_OPEN_BUNDLES = 2
CFG_POTENTIAL = 4              # the plain form computes Grav_Pot
CFG_FIND_DOMAIN = 8            # isolated: the domain is found at every decomposition
CFG_QUADRUPOLE = 16            # group form: node quadrupoles, octupole-order opening

F_TYPE, F_TIME_BIN, F_IT_DRIFT, F_IT_KICK, F_KEY, F_ID, F_COST = (1 << k for k in range(7))
F_POS, F_VEL, F_ACC, F_MASS, F_GRAV_ACC, F_LAST_ACC, F_TREE_PARENT = (1 << k for k in range(7, 14))
F_GRAV_POT = 1 << 14            # not in TVG_F_ALL

# struct Tree_Node of the reference (src/Gravity/tree.h:23-32)
TREE_DTYPE = {
    4: np.dtype([("DNext", "<i4"), ("Bitfield", "<u4"), ("DUp", "<i4"), ("Npart", "<i4"),
                 ("Pos", "<f4", 3), ("Mass", "<f4"), ("CoM", "<f4", 3), ("Dp", "<f4", 3)]),
    8: np.dtype([("DNext", "<i4"), ("Bitfield", "<u4"), ("DUp", "<i4"), ("Npart", "<i4"),
                 ("Pos", "<f8", 3), ("Mass", "<f8"), ("CoM", "<f8", 3), ("Dp", "<f8", 3)]),
}
TOPNODE_DTYPE = np.dtype([("Key", "<u8"), ("Target", "<i4"), ("Level", "<i4"),
                          ("First_Part", "<i4"), ("Npart", "<i4"), ("Pos", "<f4", 3),
                          ("Mass", "<f4"), ("CoM", "<f4", 3), ("Dp", "<f4", 3)])


class Config(C.Structure):
    _fields_ = [("float_bytes", C.c_int32), ("periodic", C.c_int32), ("boxsize", C.c_double),
                ("gravity", C.c_double), ("softening", C.c_double), ("open_bh", C.c_double),
                ("open_rel", C.c_double), ("vector_size", C.c_int32), ("flags", C.c_int32),
                ("max_particles", C.c_int64)]


class Particles(C.Structure):
    _fields_ = [("type", C.c_void_p), ("time_bin", C.c_void_p), ("it_drift_pos", C.c_void_p),
                ("it_kick_pos", C.c_void_p), ("key", C.c_void_p), ("id", C.c_void_p),
                ("cost", C.c_void_p), ("pos", C.c_void_p * 3), ("vel", C.c_void_p * 3),
                ("acc", C.c_void_p * 3), ("mass", C.c_void_p), ("grav_acc", C.c_void_p * 3),
                ("last_acc_mag", C.c_void_p), ("tree_parent", C.c_void_p), ("grav_pot", C.c_void_p)]


class TimelineConfig(C.Structure):
    _fields_ = [("comoving", C.c_int32), ("time_begin", C.c_double), ("time_end", C.c_double),
                ("hubble_constant", C.c_double), ("omega_matter", C.c_double),
                ("omega_lambda", C.c_double), ("omega_rad", C.c_double), ("omega_0", C.c_double),
                ("omega_baryon", C.c_double), ("rho_crit0", C.c_double),
                ("time_int_accuracy", C.c_double), ("max_timestep", C.c_double),
                ("displ_constraint", C.c_double)]


class TimelineState(C.Structure):
    _fields_ = [("beg", C.c_uint32), ("current", C.c_uint32), ("next", C.c_uint32),
                ("end", C.c_uint32), ("step", C.c_uint32), ("next_sync_point", C.c_uint32),
                ("time_current", C.c_double), ("time_next", C.c_double), ("time_step", C.c_double),
                ("step_max", C.c_double), ("step_min", C.c_double),
                ("expansion_factor", C.c_double), ("hubble_parameter", C.c_double),
                ("dt_max_global", C.c_float), ("max_active_bin", C.c_int32),
                ("time_bin_min", C.c_int32), ("time_bin_max", C.c_int32),
                ("sync_point", C.c_int32), ("first_step", C.c_int32), ("prepare_step", C.c_int32),
                ("n_active", C.c_int64), ("step_counter", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class MlpTrainConfig(C.Structure):
    _fields_ = [("steps", C.c_int32), ("batch", C.c_int32), ("n_samples", C.c_int64),
                ("lr", C.c_float), ("lr_final", C.c_float), ("seed", C.c_uint64),
                ("resume", C.c_int32)]


MLP_NPARAM = 4672

# optional blocks of a snapshot after POS, VEL, ID, MASS (src/IO/io.h:74-85);
# SNAP_MASS: a read found the MASS block
SNAP_ACC, SNAP_GACC, SNAP_GPOT, SNAP_MASS = 1, 2, 4, 8


class SnapshotHeader(C.Structure):
    """struct gadget_header of the reference (src/IO/io.h:24-44), less its fill."""
    _fields_ = [("npart", C.c_uint32 * 6), ("nall", C.c_uint64 * 6), ("massarr", C.c_double * 6),
                ("time", C.c_double), ("redshift", C.c_double), ("num_files", C.c_int32),
                ("boxsize", C.c_double), ("omega0", C.c_double), ("omega_lambda", C.c_double),
                ("hubble_param", C.c_double)]


def snapshot_header(npart, time, boxsize, omega0=1.0, omega_lambda=0.0, hubble_param=0.7,
                    comoving=True, nall=None, massarr=None, num_files=1):
    """Header as Write_Snapshot fills it (src/IO/write_snapshot.c:183-219).

    ``npart`` / ``nall`` are six per-type counts (an int means all type 1);
    Redshift is 1/Time - 1 for a comoving run and 0 otherwise."""
    def six(v):
        return [0, int(v), 0, 0, 0, 0] if np.isscalar(v) else [int(x) for x in v]
    h = SnapshotHeader()
    h.npart[:] = six(npart)
    h.nall[:] = six(npart if nall is None else nall)
    h.massarr[:] = [0.0] * 6 if massarr is None else [float(m) for m in massarr]
    h.time = time
    h.redshift = 1.0 / time - 1.0 if comoving else 0.0
    h.num_files = num_files
    h.boxsize, h.omega0, h.omega_lambda, h.hubble_param = boxsize, omega0, omega_lambda, hubble_param
    return h


def write_snapshot_host(path, header, pos, vel, ids, mass, acc=None, grav_acc=None,
                        grav_pot=None):
    """Write a snapshot of host arrays (tvg_write_snapshot_host): pos, vel
    (and acc, grav_acc) shaped (3, n), ids uint32, all Floats of one width."""
    ft = np.asarray(pos).dtype
    n = np.asarray(mass).shape[0]

    def f(a, shape):
        a = np.ascontiguousarray(a, dtype=ft)
        assert a.shape == shape, (a.shape, shape)
        return a

    keep = [f(pos, (3, n)), f(vel, (3, n)), np.ascontiguousarray(ids, dtype=np.uint32),
            f(mass, (n,))]
    p = Particles()
    for k in range(3):
        p.pos[k] = keep[0][k].ctypes.data
        p.vel[k] = keep[1][k].ctypes.data
    p.id, p.mass = keep[2].ctypes.data, keep[3].ctypes.data
    blocks = 0
    if acc is not None:
        keep.append(f(acc, (3, n)))
        for k in range(3):
            p.acc[k] = keep[-1][k].ctypes.data
        blocks |= SNAP_ACC
    if grav_acc is not None:
        keep.append(f(grav_acc, (3, n)))
        for k in range(3):
            p.grav_acc[k] = keep[-1][k].ctypes.data
        blocks |= SNAP_GACC
    if grav_pot is not None:
        keep.append(f(grav_pot, (n,)))
        p.grav_pot = keep[-1].ctypes.data
        blocks |= SNAP_GPOT
    rc = lib().tvg_write_snapshot_host(str(path).encode(), C.byref(header), C.c_int64(n),
                                       C.c_int32(ft.itemsize), C.byref(p), C.c_uint32(blocks))
    if rc != TVG_OK:
        raise TvgError(rc, f"tvg_write_snapshot_host({path})")


class TvgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def _ptr(a):
    return None if a is None else a.ctypes.data


class GravityContext:
    """Device context of the gravity hot path (tvg_init ... tvg_finalize)."""

    def __init__(self, max_particles, float_bytes=4, periodic=False, boxsize=0.0,
                 gravity=GRAVITY, softening=0.01, open_bh=0.25, open_rel=0.005,
                 vector_size=64, flags=0, device=0):
        self.lib = lib()
        self.fb = float_bytes
        self.ft = np.float32 if float_bytes == 4 else np.float64
        cfg = Config(float_bytes, int(periodic), boxsize, gravity, softening, open_bh, open_rel,
                     vector_size, flags, int(max_particles))
        self.cfg = cfg
        self.ctx = C.c_void_p()
        rc = self.lib.tvg_init(C.c_int(device), C.byref(cfg), C.byref(self.ctx))
        if rc != TVG_OK:
            msg = self.lib.tvg_last_error(self.ctx).decode() if self.ctx else ""
            if self.ctx:
                self.lib.tvg_finalize(self.ctx)
            self.ctx = None
            raise TvgError(rc, f"tvg_init failed {msg}")
        self.n = 0

    def close(self):
        if self.ctx:
            self.lib.tvg_finalize(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != TVG_OK:
            raise TvgError(rc, f"{what}: {self.lib.tvg_last_error(self.ctx).decode()}")

    # ------------------------------------------------------------ data

    def upload(self, pos, mass, vel=None, ids=None, last_acc=None, types=None, time_bin=None,
               it_drift=None, it_kick=None, acc=None, grav_acc=None, cost=None):
        ft = self.ft
        n = int(np.asarray(mass).shape[0])
        self._keep = []
        p = Particles()
        fields = F_POS | F_MASS
        for name, bit, arr, dt in (("type", F_TYPE, types, np.int32),
                                   ("time_bin", F_TIME_BIN, time_bin, np.int32),
                                   ("it_drift_pos", F_IT_DRIFT, it_drift, np.uint32),
                                   ("it_kick_pos", F_IT_KICK, it_kick, np.uint32)):
            if arr is not None:
                a = np.ascontiguousarray(arr, dtype=dt)
                self._keep.append(a)
                setattr(p, name, a.ctypes.data)
                fields |= bit
        for name, bit, arr in (("acc", F_ACC, acc), ("grav_acc", F_GRAV_ACC, grav_acc)):
            if arr is not None:
                fields |= bit
                dst = getattr(p, name)
                for k in range(3):
                    a = np.ascontiguousarray(arr[k], dtype=ft)
                    self._keep.append(a)
                    dst[k] = a.ctypes.data
        for k in range(3):
            a = np.ascontiguousarray(pos[k], dtype=ft)
            self._keep.append(a)
            p.pos[k] = a.ctypes.data
        m = np.ascontiguousarray(mass, dtype=ft)
        self._keep.append(m)
        p.mass = m.ctypes.data
        if vel is not None:
            fields |= F_VEL
            for k in range(3):
                a = np.ascontiguousarray(vel[k], dtype=ft)
                self._keep.append(a)
                p.vel[k] = a.ctypes.data
        ids = np.arange(n, dtype=np.uint32) if ids is None else np.ascontiguousarray(ids, np.uint32)
        self._keep.append(ids)
        p.id = ids.ctypes.data
        fields |= F_ID
        if cost is not None:          # P.Cost: what a balanced decomposition weighs
            c_arr = np.ascontiguousarray(cost, dtype=ft)
            self._keep.append(c_arr)
            p.cost = c_arr.ctypes.data
            fields |= F_COST
        la = np.zeros(n, ft) if last_acc is None else np.ascontiguousarray(last_acc, dtype=ft)
        self._keep.append(la)
        p.last_acc_mag = la.ctypes.data
        fields |= F_LAST_ACC
        self._check(self.lib.tvg_upload(self.ctx, C.c_int64(n), C.byref(p), C.c_uint32(fields)),
                    "upload")
        self.n = n

    def download(self, fields=F_POS | F_MASS | F_ID | F_ACC | F_GRAV_ACC | F_COST):
        n, ft = self.n, self.ft
        out = {}
        p = Particles()
        if fields & F_POS:
            out["pos"] = np.zeros((3, n), ft)
            for k in range(3):
                p.pos[k] = out["pos"][k].ctypes.data
        for name, bit in (("acc", F_ACC), ("grav_acc", F_GRAV_ACC), ("vel", F_VEL)):
            if fields & bit:
                out[name] = np.zeros((3, n), ft)
                arr = getattr(p, name)
                for k in range(3):
                    arr[k] = out[name][k].ctypes.data
        for name, bit, dt in (("mass", F_MASS, ft), ("cost", F_COST, ft),
                              ("last_acc_mag", F_LAST_ACC, ft), ("id", F_ID, np.uint32),
                              ("tree_parent", F_TREE_PARENT, np.int32),
                              ("grav_pot", F_GRAV_POT, ft),
                              ("time_bin", F_TIME_BIN, np.int32), ("type", F_TYPE, np.int32),
                              ("it_drift_pos", F_IT_DRIFT, np.uint32),
                              ("it_kick_pos", F_IT_KICK, np.uint32)):
            if fields & bit:
                out[name] = np.zeros(n, dt)
                setattr(p, name, out[name].ctypes.data)
        if fields & F_KEY:
            out["key"] = np.zeros((n, 2), np.uint64)
            p.key = out["key"].ctypes.data
        self._check(self.lib.tvg_download(self.ctx, C.byref(p), C.c_uint32(fields)), "download")
        if "key" in out:   # little-endian 128-bit -> [hi, lo]
            out["key"] = np.ascontiguousarray(out["key"][:, ::-1])
        return out

    # ------------------------------------------------- reference entry points

    def set_domain(self, origin, size):
        o = (C.c_double * 3)(*origin)
        self._check(self.lib.tvg_set_domain(self.ctx, o, C.c_double(size)), "set_domain")

    def find_domain(self):
        """set_computational_domain on the device (tvg_find_domain); sets and
        returns (origin, size)."""
        o = (C.c_double * 3)()
        s = C.c_double()
        self._check(self.lib.tvg_find_domain(self.ctx, o, C.byref(s)), "find_domain")
        return np.array(o[:]), s.value

    def peano_keys(self):
        self._check(self.lib.tvg_peano_keys(self.ctx), "peano_keys")

    def reverse_keys(self):
        self._check(self.lib.tvg_reverse_keys(self.ctx), "reverse_keys")

    def sort_particles(self, want_perm=True):
        perm = np.zeros(self.n, np.uint32) if want_perm else None
        self._check(self.lib.tvg_sort_particles(self.ctx, C.c_void_p(_ptr(perm))), "sort")
        return perm

    def set_domain_decomposition(self, ntask=1, part_alloc_factor=1.1, imbal_ceil=0.05):
        """Domain_Decomposition over NTask targets (tvg_set_domain_decomposition)."""
        self._check(self.lib.tvg_set_domain_decomposition(
            self.ctx, C.c_int32(ntask), C.c_double(part_alloc_factor), C.c_double(imbal_ceil)),
            "set_domain_decomposition")

    def decomposition_rounds(self):
        r = C.c_int32()
        self._check(self.lib.tvg_decomposition_rounds(self.ctx, C.byref(r)), "decomposition_rounds")
        return r.value

    def top_nodes(self):
        nt = C.c_int32()
        self._check(self.lib.tvg_top_nodes(self.ctx, C.byref(nt)), "top_nodes")
        return nt.value

    def tree_build(self, exact_moments=True):
        self._check(self.lib.tvg_tree_build(self.ctx, C.c_uint32(
            BUILD_EXACT_MOMENTS if exact_moments else 0)), "tree_build")

    def download_tree(self):
        nn = C.c_int64()
        nt = C.c_int32()
        self._check(self.lib.tvg_download_tree(self.ctx, None, C.c_int64(0), C.byref(nn), None,
                                               C.c_int32(0), C.byref(nt)), "download_tree")
        tree = np.zeros(max(nn.value, 1), TREE_DTYPE[self.fb])
        top = np.zeros(max(nt.value, 1), TOPNODE_DTYPE)
        self._check(self.lib.tvg_download_tree(self.ctx, C.c_void_p(tree.ctypes.data),
                                               C.c_int64(len(tree)), C.byref(nn),
                                               C.c_void_p(top.ctypes.data), C.c_int32(len(top)),
                                               C.byref(nt)), "download_tree")
        return tree[:nn.value].copy(), top[:nt.value].copy()

    def ewald_init(self):
        self._check(self.lib.tvg_ewald_init(self.ctx), "ewald_init")

    def download_ewald_table(self):
        m = 65 ** 3
        t = [np.zeros(m, self.ft) for _ in range(4)]
        self._check(self.lib.tvg_download_ewald_table(self.ctx, *[C.c_void_p(a.ctypes.data) for a in t]),
                    "download_ewald_table")
        return t

    def upload_ewald_table(self, fx, fy, fz, fp):
        """Raw box-unit tables as in the reference's ./ewald_tables.dat."""
        t = [np.ascontiguousarray(a, dtype=self.ft) for a in (fx, fy, fz, fp)]
        self._check(self.lib.tvg_upload_ewald_table(self.ctx, *[C.c_void_p(a.ctypes.data) for a in t]),
                    "upload_ewald_table")

    def zero_accel(self):
        self._check(self.lib.tvg_zero_accel(self.ctx), "zero_accel")

    def save_last_accel(self):
        self._check(self.lib.tvg_save_last_accel(self.ctx), "save_last_accel")

    def walk(self, form=FORM_PLAIN, use_bh=True, parts=WALK_GRAVITY, ewald_kind=EWALD_TABLE):
        self._check(self.lib.tvg_walk(self.ctx, C.c_int32(form), C.c_int32(int(use_bh)),
                                      C.c_uint32(parts), C.c_int32(ewald_kind)), "walk")

    def force_step(self, form=FORM_GROUP, use_bh=False, parts=WALK_GRAVITY,
                   ewald_kind=EWALD_TABLE):
        self._check(self.lib.tvg_force_step(self.ctx, C.c_int32(form), C.c_int32(int(use_bh)),
                                            C.c_uint32(parts), C.c_int32(ewald_kind)), "force_step")

    def phase_times(self):
        ms = (C.c_double * 8)()
        self._check(self.lib.tvg_phase_times(self.ctx, ms, C.c_int32(8)), "phase_times")
        return dict(zip(("keys", "sort", "top", "build", "walk", "ewald", "total"), list(ms)[:7]))

    def walk_counters(self):
        g, e = C.c_double(), C.c_double()
        self._check(self.lib.tvg_walk_counters(self.ctx, C.byref(g), C.byref(e)), "walk_counters")
        return g.value, e.value

    def walk_quad_interactions(self):
        """Of the last group walk's gravity interactions, those with a
        node's quadrupole (CFG_QUADRUPOLE); 0 otherwise."""
        q = C.c_double()
        self._check(self.lib.tvg_walk_quad_interactions(self.ctx, C.byref(q)),
                    "walk_quad_interactions")
        return q.value

    def set_opening(self, open_bh, open_rel):
        """TREE_OPEN_PARAM_BH (theta^2) and TREE_OPEN_PARAM_REL for later walks."""
        self._check(self.lib.tvg_set_opening(self.ctx, C.c_double(open_bh), C.c_double(open_rel)),
                    "set_opening")

    # ------------------------------------------- hierarchical time stepping

    def timeline_init(self, **kw):
        """Setup_Time_Integration (+ comoving kick/drift tables); keyword
        arguments are the TimelineConfig fields."""
        cfg = TimelineConfig(**kw)
        self._check(self.lib.tvg_timeline_init(self.ctx, C.byref(cfg)), "timeline_init")

    def kick_drift_table(self):
        a, k, d = (np.zeros(512) for _ in range(3))
        self._check(self.lib.tvg_download_kick_drift_table(
            self.ctx, C.c_void_p(_ptr(a)), C.c_void_p(_ptr(k)), C.c_void_p(_ptr(d))), "kd_table")
        return a, k, d

    def kick_drift_factors(self, it_curr, it_next):
        k, d = C.c_double(), C.c_double()
        self._check(self.lib.tvg_kick_drift_factors(self.ctx, C.c_uint32(it_curr), C.c_uint32(it_next),
                                                    C.byref(k), C.byref(d)), "kd_factors")
        return k.value, d.value

    def time_for_domain_update(self, domain_update_param=0.1):
        """Time_For_Domain_Update (src/signal.c:85-116); returns
        Sig.Domain_Update. The first call turns on the tree updates between
        rebuilds for this context."""
        flag = C.c_int32()
        self._check(self.lib.tvg_time_for_domain_update(self.ctx, C.c_double(domain_update_param),
                                                        C.byref(flag)), "time_for_domain_update")
        return bool(flag.value)

    def set_new_timesteps(self):
        self._check(self.lib.tvg_set_new_timesteps(self.ctx), "set_new_timesteps")

    def kick_first_halfstep(self):
        self._check(self.lib.tvg_kick_first_halfstep(self.ctx), "kick_first_halfstep")

    def kick_second_halfstep(self):
        self._check(self.lib.tvg_kick_second_halfstep(self.ctx), "kick_second_halfstep")

    def drift_to_sync_point(self):
        self._check(self.lib.tvg_drift_to_sync_point(self.ctx), "drift_to_sync_point")

    def timeline(self):
        st = TimelineState()
        self._check(self.lib.tvg_timeline_get(self.ctx, C.byref(st)), "timeline_get")
        return st

    def set_timeline(self, st):
        self._check(self.lib.tvg_timeline_set(self.ctx, C.byref(st)), "timeline_set")

    def rung_histogram(self):
        h = np.zeros(32, np.int32)
        self._check(self.lib.tvg_rung_histogram(self.ctx, C.c_void_p(_ptr(h))), "rung_histogram")
        return h

    def compute_acceleration(self, form=FORM_GROUP, parts=WALK_GRAVITY, ewald_kind=EWALD_TABLE,
                             prepare=False):
        self._check(self.lib.tvg_compute_acceleration(self.ctx, C.c_int32(form), C.c_uint32(parts),
                                                      C.c_int32(ewald_kind), C.c_int32(int(prepare))),
                    "compute_acceleration")

    def step_graph(self, parts=WALK_GRAVITY, ewald_kind=EWALD_TABLE):
        """compute_acceleration (group form, no prepare pass) as one CUDA
        graph launch; the first call of a configuration runs directly."""
        self._check(self.lib.tvg_step_graph(self.ctx, C.c_uint32(parts), C.c_int32(ewald_kind)),
                    "step_graph")

    def step_graph_reset(self):
        self._check(self.lib.tvg_step_graph_reset(self.ctx), "step_graph_reset")

    def autotune(self, use_bh=False, parts=WALK_GRAVITY, ewald_kind=EWALD_TABLE):
        """Chooses the group size of the group form (1, 2 or 4 targets per lane)
        by timing the walks on the current tree; returns (choice, [ms1, ms2, ms4])."""
        ch = C.c_int32()
        ms = (C.c_double * 3)()
        self._check(self.lib.tvg_autotune(self.ctx, C.c_int32(int(use_bh)), C.c_uint32(parts),
                                          C.c_int32(ewald_kind), C.byref(ch), ms), "autotune")
        return ch.value, [ms[0], ms[1], ms[2]]

    # ------------------------------------------ learned Ewald correction

    def mlp_train(self, steps=4000, batch=16384, n_samples=1 << 20, lr=3e-3, lr_final=1e-5,
                  seed=1, resume=False):
        cfg = MlpTrainConfig(steps, batch, n_samples, lr, lr_final, seed, int(resume))
        loss = C.c_float()
        self._check(self.lib.tvg_ewald_mlp_train(self.ctx, C.byref(cfg), C.byref(loss)), "mlp_train")
        return loss.value

    def mlp_weights(self, params=None):
        if params is None:
            out = np.zeros(MLP_NPARAM, np.float32)
            self._check(self.lib.tvg_ewald_mlp_weights(self.ctx, C.c_void_p(_ptr(out)), C.c_int32(0)),
                        "mlp_weights")
            return out
        p = np.ascontiguousarray(params, np.float32)
        self._check(self.lib.tvg_ewald_mlp_weights(self.ctx, C.c_void_p(_ptr(p)), C.c_int32(1)),
                    "mlp_weights")

    def mlp_grad(self, x, y):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        g = np.zeros(MLP_NPARAM, np.float32)
        loss = C.c_float()
        self._check(self.lib.tvg_ewald_mlp_grad(self.ctx, C.c_int64(len(x)), C.c_void_p(_ptr(x)),
                                                C.c_void_p(_ptr(y)), C.c_void_p(_ptr(g)),
                                                C.byref(loss)), "mlp_grad")
        return g, loss.value

    def mlp_eval(self, x):
        x = np.ascontiguousarray(x, np.float64)
        t = np.zeros_like(x)
        self._check(self.lib.tvg_ewald_mlp_eval(self.ctx, C.c_int64(len(x)), C.c_void_p(_ptr(x)),
                                                C.c_void_p(_ptr(t))), "mlp_eval")
        return t

    def mlp_validate(self, max_allowed=1e-2):
        mx, rms = C.c_double(), C.c_double()
        self._check(self.lib.tvg_ewald_mlp_validate(self.ctx, C.c_double(max_allowed), C.byref(mx),
                                                 C.byref(rms)), "mlp_validate")
        return mx.value, rms.value

    def set_ewald_opening(self, rel_alpha=2.5e-4, bh_factor=0.5):
        """Opening of the group form's Ewald walk (see tvg_set_ewald_opening)."""
        self._check(self.lib.tvg_set_ewald_opening(self.ctx, C.c_double(rel_alpha),
                                                   C.c_double(bh_factor)), "set_ewald_opening")

    def set_walk_limit(self, max_iterations=1 << 24):
        """Iteration limit of the group walks (see tvg_set_walk_limit)."""
        self._check(self.lib.tvg_set_walk_limit(self.ctx, C.c_int64(max_iterations)),
                    "set_walk_limit")

    def forcetest(self, targets, parts=None):
        """Gravity_Forcetest: FP64 direct force on the targets (sorted-order
        indices), Ewald-summed when ``parts`` has WALK_EWALD (default: when
        periodic). Returns (a_direct (3, nt), a_tree (3, nt), {"rms", "p99",
        "mean", "max"} of the relative error)."""
        if parts is None:
            parts = WALK_GRAVITY | (WALK_EWALD if self.cfg.periodic else 0)
        t = np.ascontiguousarray(targets, dtype=np.int64)
        nt = len(t)
        ad = np.empty((3, nt), np.float64)
        at = np.empty((3, nt), np.float64)
        err = np.empty(4, np.float64)
        self._check(self.lib.tvg_forcetest(self.ctx, C.c_uint32(parts), C.c_int64(nt),
                                           C.c_void_p(_ptr(t)),
                                           C.c_void_p(_ptr(ad)), C.c_void_p(_ptr(at)),
                                           C.c_void_p(_ptr(err))), "forcetest")
        return ad, at, dict(zip(("rms", "p99", "mean", "max"), map(float, err)))

    # ------------------------------------------------ active set, timing

    def set_active(self, indices=None):
        """Active_Particle_List (sorted-order indices); None = all particles."""
        if indices is None:
            self._check(self.lib.tvg_set_active(self.ctx, None, C.c_int64(0)), "set_active")
            return
        a = np.ascontiguousarray(indices, dtype=np.int32)
        self._check(self.lib.tvg_set_active(self.ctx, C.c_void_p(a.ctypes.data), C.c_int64(len(a))),
                    "set_active")

    def timer_start(self):
        self._check(self.lib.tvg_timer(self.ctx, C.c_int32(0), None), "timer")

    def timer_stop(self):
        ms = C.c_double()
        self._check(self.lib.tvg_timer(self.ctx, C.c_int32(1), C.byref(ms)), "timer")
        return ms.value

    def launch_count(self):
        n = C.c_int64()
        self._check(self.lib.tvg_launch_count(self.ctx, C.byref(n)), "launch_count")
        return n.value

    def fp32_peak(self, ms_target=200.0):
        t = C.c_double()
        self._check(self.lib.tvg_fp32_peak(self.ctx, C.c_double(ms_target), C.byref(t)), "fp32_peak")
        return t.value

    def upload_fields(self, n, pos=None, mass=None, last_acc=None, ids=None):
        """Upload pre-allocated (e.g. pinned) Float arrays without copies."""
        p = Particles()
        fields = 0
        if ids is not None:
            p.id = ids.ctypes.data
            fields |= F_ID
        if pos is not None:
            for k in range(3):
                p.pos[k] = pos[k].ctypes.data
            fields |= F_POS
        if mass is not None:
            p.mass = mass.ctypes.data
            fields |= F_MASS
        if last_acc is not None:
            p.last_acc_mag = last_acc.ctypes.data
            fields |= F_LAST_ACC
        self._check(self.lib.tvg_upload(self.ctx, C.c_int64(n), C.byref(p), C.c_uint32(fields)),
                    "upload")
        self.n = n

    def read_snapshot(self, path):
        """Read_Snapshot onto the device (tvg_read_snapshot); returns the
        particle count and the optional blocks found."""
        n, b = C.c_int64(), C.c_uint32()
        self._check(self.lib.tvg_read_snapshot(self.ctx, str(path).encode(), C.byref(n), C.byref(b)),
                    "read_snapshot")
        self.n = n.value
        return n.value, b.value

    def write_snapshot(self, path, header, blocks=0):
        """Write_Snapshot of the resident particles in their device order."""
        self._check(self.lib.tvg_write_snapshot(self.ctx, str(path).encode(), C.byref(header),
                                                C.c_uint32(blocks)), "write_snapshot")

    def download_into(self, grav_acc=None, ids=None):
        """Download into pre-allocated (e.g. pinned) arrays."""
        p = Particles()
        fields = 0
        if grav_acc is not None:
            for k in range(3):
                p.grav_acc[k] = grav_acc[k].ctypes.data
            fields |= F_GRAV_ACC
        if ids is not None:
            p.id = ids.ctypes.data
            fields |= F_ID
        self._check(self.lib.tvg_download(self.ctx, C.byref(p), C.c_uint32(fields)), "download")

    def force_step_host(self, n, pos, mass, last_acc=None, ids=None, grav_acc=None, ids_out=None,
                        form=FORM_GROUP, use_bh=False, parts=WALK_GRAVITY, ewald_kind=EWALD_TABLE):
        """tvg_force_step_host: one force step from pre-allocated (e.g.
        pinned) Float arrays, results (PH order) into grav_acc / ids_out."""
        src, dst = Particles(), Particles()
        fin = F_POS | F_MASS
        for k in range(3):
            src.pos[k] = pos[k].ctypes.data
        src.mass = mass.ctypes.data
        if last_acc is not None:
            src.last_acc_mag = last_acc.ctypes.data
            fin |= F_LAST_ACC
        if ids is not None:
            src.id = ids.ctypes.data
            fin |= F_ID
        fout = 0
        if grav_acc is not None:
            for k in range(3):
                dst.grav_acc[k] = grav_acc[k].ctypes.data
            fout |= F_GRAV_ACC
        if ids_out is not None:
            dst.id = ids_out.ctypes.data
            fout |= F_ID
        self._check(self.lib.tvg_force_step_host(self.ctx, C.c_int64(n), C.byref(src), C.c_uint32(fin),
                                                 C.byref(dst), C.c_uint32(fout), C.c_int32(form),
                                                 C.c_int32(int(use_bh)), C.c_uint32(parts),
                                                 C.c_int32(ewald_kind)), "force_step_host")
        self.n = n


def read_snapshot_header(path):
    """The header of a snapshot (or of path.0 of a split one) and the number
    of files (tvg_read_snapshot_header)."""
    h = SnapshotHeader()
    nf = C.c_int32()
    rc = lib().tvg_read_snapshot_header(str(path).encode(), C.byref(h), C.byref(nf))
    if rc != TVG_OK:
        raise TvgError(rc, f"tvg_read_snapshot_header({path})")
    return h, nf.value


def read_snapshot(path, float_bytes=4):
    """Read_Snapshot into numpy arrays (tvg_read_snapshot_host): pos, vel
    (3, n), id, mass, type, and acc0, grav_acc, grav_pot when the file has
    them; the particles in the reference's order (type sections, each in
    file order)."""
    h, nf = read_snapshot_header(path)
    cap = int(sum(h.nall))
    ft = np.float32 if float_bytes == 4 else np.float64
    a = dict(pos=np.zeros((3, cap), ft), vel=np.zeros((3, cap), ft), id=np.zeros(cap, np.uint32),
             mass=np.zeros(cap, ft), type=np.zeros(cap, np.int32), acc0=np.zeros(cap, ft),
             grav_acc=np.zeros((3, cap), ft), grav_pot=np.zeros(cap, ft))
    p = Particles()
    for k in range(3):
        p.pos[k] = a["pos"][k].ctypes.data
        p.vel[k] = a["vel"][k].ctypes.data
        p.grav_acc[k] = a["grav_acc"][k].ctypes.data
    p.acc[0] = a["acc0"].ctypes.data
    p.id, p.mass, p.type = a["id"].ctypes.data, a["mass"].ctypes.data, a["type"].ctypes.data
    p.grav_pot = a["grav_pot"].ctypes.data
    n, blocks = C.c_int64(), C.c_uint32()
    rc = lib().tvg_read_snapshot_host(str(path).encode(), C.c_int32(float_bytes), C.c_int64(cap),
                                      C.byref(p), C.byref(n), C.byref(blocks))
    if rc != TVG_OK:
        raise TvgError(rc, f"tvg_read_snapshot_host({path})")
    m, b = n.value, blocks.value
    out = {k: v[..., :m] for k, v in a.items()}
    for name, bit in (("acc0", SNAP_ACC), ("grav_acc", SNAP_GACC), ("grav_pot", SNAP_GPOT)):
        if not b & bit:
            del out[name]
    out.update(header=h, num_files=nf, n=m, blocks=b)
    return out


def host_register(a):
    """Page-lock the memory of a contiguous numpy array (tvg_host_register)."""
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("host_register needs a contiguous array")
    rc = lib().tvg_host_register(C.c_void_p(a.ctypes.data), C.c_size_t(a.nbytes))
    if rc != TVG_OK:
        raise TvgError(rc, "tvg_host_register failed")


def host_unregister(a):
    """Release a range registered with host_register."""
    rc = lib().tvg_host_unregister(C.c_void_p(a.ctypes.data))
    if rc != TVG_OK:
        raise TvgError(rc, "tvg_host_unregister failed")


class PinnedArray:
    """numpy view of page-locked host memory (tvg_host_alloc)."""

    def __init__(self, shape, dtype):
        self.lib = lib()
        self.nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
        self.ptr = C.c_void_p()
        rc = self.lib.tvg_host_alloc(C.c_size_t(self.nbytes), C.byref(self.ptr))
        if rc != TVG_OK:
            raise TvgError(rc, "tvg_host_alloc failed")
        buf = (C.c_char * self.nbytes).from_address(self.ptr.value)
        self.array = np.frombuffer(buf, dtype=dtype).reshape(shape)

    def free(self):
        if self.ptr:
            self.array = None
            self.lib.tvg_host_free(self.ptr)
            self.ptr = None
