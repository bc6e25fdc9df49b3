#!/usr/bin/env python3
"""Tree-force throughput of the Tandav gravity hot path on B200.

Workload (the reference's headline configuration, synthetic): a periodic
cosmological box of 256^3 particles, 100 Mpc/h, Zel'dovich displacements at
z = 50 from a seeded Gaussian field (Eisenstein & Hu 1998 P(k)), softening
1/30 of the mean spacing. One step = one tree-force evaluation of all
particles: Peano-Hilbert keys, sort of every particle field, top nodes, tree
build, the gravity walk with the relative opening criterion (|a_old| from an
untimed Barnes-Hut prepare pass, as src/accel.c:51-71 does) and the Ewald
periodic correction.

Our arm: the group form (FP32 integer-offset walk, warp per PH group, node
quadrupoles with the octupole-order relative criterion, a per-group Ewald
walk on a Taylor table) at TREE_OPEN_PARAM_REL 8e-3, which keeps the rms
force error below 1e-3 with a quarter in reserve (measured in every run
against an FP64 Ewald-summed direct sum over all particles for 10^4 random
particles); the step is one captured CUDA graph with the particles resident
in HBM (`value`), and the same step through the C ABI from and to pinned host
buffers with the copies overlapped (`e2e`, tvg_force_step_host). Beside it:
the plain GPU form (the reference algorithm, one thread per particle, FP64,
exact moments, the reference's TREE_OPEN_PARAM_REL 0.005) over all particles
with its own measured error, the group form at the plain form's opening, the
group form with monopoles, and the learned Ewald correction.
`--impl reference`: the unmodified reference C code (oracle/_ref timing
build) on the host cores, the walk timed on a strided subset.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
       (for N > 1 launched by torch.distributed.run, one independent replica
        per GPU: the path has no data-path collective on one GPU's box)
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "tree-force particles/s at 256^3 periodic: chosen vs plain GPU form @≤1e-3 rms err"
UNIT = "particles/s"
# flop counted per interaction (a fixed convention shared by both forms):
# monopole / particle pair = 3 sub, 5 for r^2, rsqrt, 2 for r^-3, mass,
# 6 for the accumulation, 2 for the criterion; table Ewald = fold and three
# 8-corner trilinear interpolations
FLOP_PER_GRAV = 20.0
FLOP_PER_EWALD = 60.0
# node quadrupole (group form, --quadrupole): 3 sub, 5 for r^2, rsqrt, 4 for
# r^-3, r^-5, r^-7, mass, 15 for Q d, 5 for d.Q d, 3 for the radial factor,
# 12 for the accumulation, 2 for the criterion
FLOP_PER_QUAD = 51.0
CFG_QUADRUPOLE = 16
# operating points (TREE_OPEN_PARAM_REL, Ewald alpha_E) at 256^3, the fastest
# of a sweep that keeps the rms force error below 1e-3 with margin:
# quadrupoles (the headline) and the reference's monopoles (9.7e-4)
QUAD_OPEN = (8e-3, 1e-2)
MONO_OPEN = (7e-5, 4e-4)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nside", type=int, default=256)
    ap.add_argument("--box-mpc", type=float, default=100.0, help="box side, Mpc/h")
    ap.add_argument("--tpl", type=int, default=0, choices=[0, 1, 2, 4],
                    help="targets per lane of the group walk (0: autotune)")
    ap.add_argument("--plain-stride", type=int, default=1,
                    help="walk every s-th particle in the plain form (1: all particles, no "
                         "extrapolation)")
    ap.add_argument("--no-matched", action="store_true",
                    help="skip the group form at the plain form's opening parameter")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-mlp", action="store_true", help="skip the learned-Ewald step")
    ap.add_argument("--no-peak", action="store_true", help="skip the FFMA peak loop (profiling runs)")
    ap.add_argument("--monopole", action="store_true",
                    help="headline group form with node monopoles (the reference's moments) "
                         "instead of quadrupoles (TVG_CFG_QUADRUPOLE)")
    ap.add_argument("--open-rel", type=float, default=None,
                    help="TREE_OPEN_PARAM_REL of the headline group form (default: the operating "
                         "point of its form, QUAD_OPEN or MONO_OPEN)")
    ap.add_argument("--ewald-alpha", type=float, default=None,
                    help="opening of the group form's Ewald walk, relative to |a_old| (default: "
                         "the operating point of its form)")
    ap.add_argument("--vector-size", type=int, default=32,
                    help="VECTOR_SIZE of the headline form's tree: particles per bundle (the "
                         "reference's default is 64; 32 gives smaller bundles near each group, "
                         "41 %% fewer interactions at the same force error)")
    ap.add_argument("--no-monopole-run", action="store_true",
                    help="skip the monopole group form's own run (quadrupole headline only)")
    ap.add_argument("--plain-open-rel", type=float, default=0.005,
                    help="TREE_OPEN_PARAM_REL of the plain form (the reference's value)")
    ap.add_argument("--domain-update-param", type=float, default=None,
                    help="rung run: follow Time_For_Domain_Update with this DOMAIN_UPDATE_PARAM "
                         "(the reference's 0.1), keeping and updating the tree between domain "
                         "updates; default: rebuild at every step")
    ap.add_argument("--rung-steps", type=int, default=0,
                    help="also run this many hierarchical time steps from z = 50 (rung workload)")
    ap.add_argument("--time-int-accuracy", type=float, default=0.025)
    ap.add_argument("--forcetest-targets", type=int, default=10000,
                    help="particles in the FP64 direct-sum error check (0: skip)")
    args = ap.parse_args()
    rel, alpha = MONO_OPEN if args.monopole else QUAD_OPEN
    args.open_rel = rel if args.open_rel is None else args.open_rel
    args.ewald_alpha = alpha if args.ewald_alpha is None else args.ewald_alpha
    args.flags = 0 if args.monopole else CFG_QUADRUPOLE
    return args


def dist_info():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Dist:
    """Barrier and max over ranks (gloo on host tensors); a no-op at N = 1."""

    def __init__(self, ws):
        self.ws = ws
        if ws > 1:
            import datetime
            import torch.distributed as td
            td.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
            self.td = td

    def barrier(self):
        if self.ws > 1:
            self.td.barrier()

    def max(self, v):
        if self.ws == 1:
            return v
        import torch
        t = torch.tensor([float(v)], dtype=torch.float64)
        self.td.all_reduce(t, op=self.td.ReduceOp.MAX)
        return float(t.item())

    def sum(self, v):
        if self.ws == 1:
            return v
        import torch
        t = torch.tensor([float(v)], dtype=torch.float64)
        self.td.all_reduce(t, op=self.td.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.ws > 1:
            self.td.destroy_process_group()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.gpu)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.t:
            self.t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def make_ics(nside, seed, box_mpc=100.0):
    from tandav_b200 import ics
    return ics.zeldovich_box(n_side=nside, box_mpc=box_mpc, seed=seed)


def device_memory_used_gb(index):
    """Device memory in use on the GPU (NVML), GB."""
    try:
        import pynvml
        pynvml.nvmlInit()
        try:
            h = pynvml.nvmlDeviceGetHandleByIndex(index)
            return round(pynvml.nvmlDeviceGetMemoryInfo(h).used / 1e9, 2)
        finally:
            pynvml.nvmlShutdown()
    except Exception:         # no NVML on the host: not reported
        return None


def cpu_reference(p, cores, target_s=20.0, steps=1, warmup=0):
    """The reference's OpenMP path (oracle/_ref/per_f32_t) on strided samples
    of active particles. One run decomposes the domain and builds the tree
    for all particles, then walks warmup + steps disjoint samples (particles
    i with i % stride == r); a step is the decomposition, the build and one
    sample's relative walk extrapolated to all particles. Returns the mean
    over the timed steps."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import refrun
    if not refrun.available("per_f32_t"):
        return None, "reference timing build missing (make -C oracle ref)"
    if steps + warmup > 127:                 # the harness takes at most 127 samples
        warmup = min(warmup, 3)
        steps = 127 - warmup
    reps = steps + warmup
    # ~4 ms of one core per particle for the relative walk at this size: all
    # samples together take about target_s
    stride = max(8, int(p.n * 4e-3 * reps / (target_s * cores)))
    stride = max(1 << int(round(math.log2(stride))), 1 << int(math.ceil(math.log2(reps))))
    t0 = time.time()
    r = refrun.run("per_f32_t", "force", p.pos, p.vel, p.mass, box=p.box, softening=p.softening,
                   flags=3 | 4 | (stride << 8) | (reps << 24), threads=cores, timeout=3000)
    wall = time.time() - t0
    tm = r["timings"]      # ewald_init, dd, build, bh, bh_ew, rel, rel_ew, threads
    rel = r["rel_times"]
    per_step = [tm[1] + tm[2] + rel[k] * (p.n / len(range(k, p.n, stride))) for k in range(warmup, reps)]
    t_step = statistics.mean(per_step)
    n_sample = len(range(0, p.n, stride))
    return {
        "value": p.n / t_step, "unit": UNIT, "cores": int(tm[7]), "kind": "reference",
        "steps": steps, "warmup": warmup, "ms_per_step": t_step * 1e3,
        "sample": (f"unmodified reference (per_f32 timing build, -O3 -march=x86-64-v3) on the "
                   f"same {p.n}-particle box: domain decomposition {tm[1]:.2f} s and tree build "
                   f"{tm[2]:.2f} s for all particles; per step the relative-criterion walk incl. "
                   f"Ewald of every {stride}th particle (~{n_sample}, a different offset each "
                   f"step, {warmup} untimed), mean {statistics.mean(rel[warmup:]):.2f} s, "
                   f"extrapolated linearly to all; run wall {wall:.0f} s"),
    }, None


def run_reference_arm(args):
    ws, rank, _ = dist_info()
    if rank != 0:
        return 0
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    p = make_ics(args.nside, 1234, args.box_mpc)
    try:
        cb, err = cpu_reference(p, cores, target_s=60.0, steps=args.steps, warmup=args.warmup)
    except Exception as e:           # a failed or timed-out reference run
        cb, err = None, f"reference run failed: {e}"
    if cb is None:
        print(json.dumps({"impl": "reference", "unavailable": err}))
        return 0
    out = {
        "impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": 0,
        "steps": cb["steps"], "warmup": cb["warmup"], "ms_per_step": cb["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded Zel'dovich box (see config)",
        "config": workload_config(args, p, ws),
        "cpu_baseline": cb,
        "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


def rung_run(args, p, G, device):
    """Hierarchical time stepping from z = 50 (src/main.c:43-70): per step
    Set_New_Timesteps, first kick, drift, Compute_Acceleration of the active
    particles, second kick; per-step active particles, time and rung counts."""
    ctx = G.GravityContext(p.n, float_bytes=4, periodic=True, boxsize=p.box, softening=p.softening,
                           device=device, flags=args.flags)
    try:
        n = p.n
        ctx.upload(p.pos, p.mass, vel=p.vel, types=np.ones(n, np.int32),
                   time_bin=np.zeros(n, np.int32), it_drift=np.zeros(n, np.uint32),
                   it_kick=np.zeros(n, np.uint32))
        ctx.set_domain((0.0, 0.0, 0.0), p.box)
        ctx.ewald_init()
        ctx.set_opening(0.25, args.open_rel)
        ctx.set_ewald_opening(args.ewald_alpha)
        h0 = 0.1
        ctx.timeline_init(comoving=1, time_begin=p.a_start, time_end=1.0, hubble_constant=h0,
                          omega_matter=0.3, omega_lambda=0.7, omega_rad=0.0, omega_0=1.0,
                          omega_baryon=0.0, rho_crit0=3 * h0 * h0 / (8 * math.pi * 43020.0),
                          time_int_accuracy=args.time_int_accuracy, max_timestep=0.05,
                          displ_constraint=0.25)
        parts = G.WALK_GRAVITY | G.WALK_EWALD
        ctx.timer_start()
        ctx.compute_acceleration(form=G.FORM_GROUP, parts=parts, prepare=True)
        prep_ms = ctx.timer_stop()
        dup = args.domain_update_param
        if dup is not None:
            ctx.time_for_domain_update(dup)          # Update(BEFORE_MAIN_LOOP)
        tpl = args.tpl or ctx.autotune(use_bh=False, parts=parts)[0]
        steps = []
        for _ in range(args.rung_steps):
            st = ctx.timeline()
            if st.current >= st.end:
                break
            # each phase in its own device-timed region (events on the
            # library stream); the step's time is their sum
            ctx.timer_start()
            ctx.set_new_timesteps()
            bins_ms = ctx.timer_stop()
            st = ctx.timeline()
            ctx.timer_start()
            ctx.kick_first_halfstep()
            kick1_ms = ctx.timer_stop()
            ctx.timer_start()
            ctx.drift_to_sync_point()
            drift_ms = ctx.timer_stop()
            rebuilt = ctx.time_for_domain_update(dup) if dup is not None else True
            ctx.timer_start()
            ctx.step_graph(parts)              # Compute_Acceleration, one graph launch
            force_ms = ctx.timer_stop()
            ctx.timer_start()
            ctx.kick_second_halfstep()
            kick2_ms = ctx.timer_stop()
            ms = bins_ms + kick1_ms + drift_ms + force_ms + kick2_ms
            h = ctx.rung_histogram()
            ph = ctx.phase_times()
            g_i, e_i = ctx.walk_counters()
            steps.append({"a": round(st.time_current, 6), "n_active": int(st.n_active),
                          "max_active_bin": int(st.max_active_bin), "rebuilt": bool(rebuilt),
                          "ms": round(ms, 2),
                          "timesteps_ms": round(bins_ms, 3), "kick_ms": round(kick1_ms + kick2_ms, 3),
                          "drift_ms": round(drift_ms, 3), "force_ms": round(force_ms, 2),
                          "walk_ms": round(ph["walk"], 1), "ewald_ms": round(ph["ewald"], 1),
                          "interactions_per_active": round(g_i / max(st.n_active, 1)),
                          "ewald_evals_per_active": round(e_i / max(st.n_active, 1), 1),
                          "particles_per_s": round(st.n_active / (ms * 1e-3)),
                          "rungs": {int(b): int(c) for b, c in enumerate(h) if c}})
        tot_ms = sum(s["ms"] for s in steps)
        tot_act = sum(s["n_active"] for s in steps)
        # kick and drift against the copy bandwidth, over the steps that move
        # every particle: 36 B per particle and kick or drift (Vel += dt Acc;
        # Pos += dt Vel, FP32), the kernels' own traffic 48 B per kick (also
        # Time_Bin and It_Kick_Pos) and 44 B per drift (It_Drift_Pos)
        full = [s for s in steps if s["n_active"] == n and s["rebuilt"]]
        hbm = None
        if full:
            k_ms = min(s["kick_ms"] for s in full) / 2.0
            d_ms = min(s["drift_ms"] for s in full)
            hbm = {"steps": len(full), "n_particles": n,
                   "kick_ms": round(k_ms, 4), "drift_ms": round(d_ms, 4),
                   "kick_gbs_algorithmic": round(36.0 * n / (k_ms * 1e6), 1),
                   "drift_gbs_algorithmic": round(36.0 * n / (d_ms * 1e6), 1),
                   "kick_gbs_touched": round(48.0 * n / (k_ms * 1e6), 1),
                   "drift_gbs_touched": round(44.0 * n / (d_ms * 1e6), 1),
                   "timing": "fastest full step; one half kick is half the step's two kicks"}
        return {"workload": f"zeldovich_{args.nside}^3 from z = 50, hierarchical steps, "
                            f"TimeIntAccuracy {args.time_int_accuracy}",
                "tree": ("rebuilt every step" if dup is None else
                         f"kept between domain updates, DOMAIN_UPDATE_PARAM {dup}"),
                "prepare_ms": round(prep_ms, 1), "targets_per_lane": tpl,
                "steps": len(steps), "total_ms": round(tot_ms, 1),
                "active_particles_per_s": round(tot_act / (tot_ms * 1e-3)) if tot_ms else None,
                "rungs_populated_max": max(len(s["rungs"]) for s in steps) if steps else 0,
                "kick_drift_hbm": hbm,
                "per_step": steps}
    finally:
        ctx.close()


def force_error(ctx, G, n, tgt_ids):
    """rms / p99 / mean / max relative force error of the particles tgt_ids
    (input order) against the FP64 direct Ewald sum on the GPU."""
    try:
        ids = ctx.download(G.F_ID)["id"]
        inv = np.empty(n, np.int64)
        inv[ids] = np.arange(n)
        _, _, err = ctx.forcetest(np.sort(inv[tgt_ids]))
        return {k: float(f"{v:.4e}") for k, v in err.items()}
    except Exception as e:
        return {"error": str(e)}


def graph_steps(ctx, parts, steps, open_rel, dist, n, G, tgt_ids, prep_err=None):
    """`steps` timed graph steps of ctx at TREE_OPEN_PARAM_REL open_rel (after a
    direct step and the two captures), with the force error of the last one.
    Every rank takes the same collective steps, failed or not."""
    err, ms, g = prep_err, math.inf, 0.0
    if err is None:
        try:
            ctx.set_opening(0.25, open_rel)
            for _ in range(3):                     # direct step, then the two captures
                ctx.step_graph(parts)
            ms = 0.0
            for _ in range(steps):
                ctx.timer_start()
                ctx.step_graph(parts)
                ms += ctx.timer_stop()
            g, _ = ctx.walk_counters()
        except Exception as e:
            err, ms = str(e), math.inf
    t = dist.max(ms / steps) / 1e3
    n_all = dist.sum(n)
    if err is not None or not math.isfinite(t):
        return {"error": err or "failed on another rank"}
    out = {"open_rel": open_rel, "particles_per_s": n_all / t, "ms_per_step": round(t * 1e3, 2),
           "steps": steps, "interactions_per_particle": round(g / n, 1)}
    if tgt_ids is not None:
        out["force_error"] = force_error(ctx, G, n, tgt_ids)
    return out


def workload_config(args, p, ws):
    return {
        "workload": f"zeldovich_{args.nside}^3_periodic_z50",
        "n_particles": int(p.n), "box_mpc_h": args.box_mpc, "z_start": 50.0,
        "softening_kpc_h": round(float(p.softening), 4),
        "criterion": (f"relative, TREE_OPEN_PARAM_REL {args.open_rel:g} (group form), "
                      f"{args.plain_open_rel:g} (plain form); |a_old| first from a BH (theta^2 "
                      f"0.25) pass"),
        "ewald_headline": ("Taylor table (the faster evaluator at the same force error); the "
                           "learned correction runs the same step in learned_ewald"),
        "ewald": (f"group form: per-group Ewald walk, Taylor table of the lattice sum (33^3 nodes, "
                  f"third order; K, dK, d2K at node centres of mass, second-order expansion about "
                  f"the group centre plus the uniform-cube remainder, a degree-7 fit of its closed "
                  f"form), opening "
                  f"alpha_E {args.ewald_alpha:g}; plain form: the reference's Ewald walk, 65^3 "
                  f"table, trilinear"),
        "form": ("group: warp per PH group of 32 x (targets per lane, autotuned) particles, FP32 on "
                 "32-bit integer box offsets"),
        "vector_size": getattr(args, "vector_size", 64),
        "moments": ("monopoles (the reference's)" if args.monopole else
                    "quadrupoles (TVG_CFG_QUADRUPOLE): every accepted node's traceless quadrupole in "
                    "the gravity walk, with the octupole-order relative criterion M s^3 <= r^5 "
                    "|a_old| TREE_OPEN_PARAM_REL / G, and in the Ewald walk's expansion"),
        "step": ("Compute_Acceleration (keys, sort, top nodes, build, |a_old|, gravity and Ewald "
                 "walks) as one captured CUDA graph launch (tvg_step_graph); |a_old| from the "
                 "previous step"),
        "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU",
        "l2": f"inputs larger than L2 ({p.n / 1e6:.1f}M particles, ~{p.n * 120 / 1e9:.1f} GB of particle state)",
    }


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)
    ws, rank, local = dist_info()
    dist = Dist(ws)
    if args.tpl:
        os.environ["TVG_GROUP_TPL"] = str(args.tpl)
    from tandav_b200 import gravity as G

    p = make_ics(args.nside, 1234 + rank, args.box_mpc)
    n = p.n
    ctx = G.GravityContext(n, float_bytes=4, periodic=True, boxsize=p.box, softening=p.softening,
                           device=local, flags=args.flags, vector_size=args.vector_size)
    parts = G.WALK_GRAVITY | G.WALK_EWALD
    ctx.upload(p.pos, p.mass)
    ctx.set_domain((0.0, 0.0, 0.0), p.box)
    ctx.ewald_init()
    ctx.set_ewald_opening(args.ewald_alpha)
    fp32_peak = 0.0 if args.no_peak else ctx.fp32_peak(ms_target=1500.0)

    # prepare step (accel.c:51-71): BH pass, |a| -> Last_Acc_Mag
    ctx.force_step(form=G.FORM_GROUP, use_bh=True, parts=parts)
    ctx.save_last_accel()
    ctx.set_opening(0.25, args.open_rel)
    ctx.force_step(form=G.FORM_GROUP, use_bh=False, parts=parts)
    if args.tpl:              # group size fixed (TVG_GROUP_TPL, set before the first walk)
        tune_choice, tune_ms = args.tpl, None
    else:
        tune_choice, tune_ms = ctx.autotune(use_bh=False, parts=parts)
    # warm-up: the first graph step runs directly, the next two capture the
    # step for the two buffer states the sort alternates between
    for _ in range(max(args.warmup, 3)):
        ctx.step_graph(parts)

    # ---- device-resident timed region
    clocks = ClockSampler(local)
    dist.barrier()
    clocks.start()
    l0 = ctx.launch_count()
    ctx.timer_start()
    walk_ms, ew_ms, grav_i, ew_i, quad_i, phases = 0.0, 0.0, 0.0, 0.0, 0.0, []
    for _ in range(args.steps):
        ctx.step_graph(parts)                  # the whole step: one CUDA graph launch
        ph = ctx.phase_times()
        phases.append(ph)
        walk_ms += ph["walk"]
        ew_ms += ph["ewald"]
        g, e = ctx.walk_counters()
        grav_i += g
        ew_i += e
        quad_i += ctx.walk_quad_interactions()
    total_ms = ctx.timer_stop()
    launches = ctx.launch_count() - l0
    clk = clocks.stop()
    hbm_gb = device_memory_used_gb(local)
    dist.barrier()
    t_step = dist.max(total_ms / args.steps) / 1e3
    value = dist.sum(n) / t_step

    # ---- force error of the timed step against the FP64 direct (Ewald) sum
    ids = G.PinnedArray((n,), np.uint32)
    ctx.download_into(ids=ids.array)
    tgt_ids = None
    accuracy = None
    if args.forcetest_targets > 0:
        nt = min(args.forcetest_targets, n)
        tgt_ids = np.sort(np.random.default_rng(777).choice(n, nt, replace=False))
        inv = np.empty(n, np.int64)
        inv[ids.array] = np.arange(n)
        try:
            ctx.timer_start()
            _, _, err = ctx.forcetest(np.sort(inv[tgt_ids]))
            ft_ms = ctx.timer_stop()
            accuracy = {"targets": int(nt), "group": {k: float(f"{v:.4e}") for k, v in err.items()},
                        "oracle": "FP64 direct sum on the GPU over all particles, softened kernel, "
                                  "Ewald-summed (alpha L = 12, nearest-image real space, |h|^2 <= 576)",
                        "forcetest_ms": round(ft_ms, 1)}
        except Exception as e:       # the headline line is printed all the same
            accuracy, tgt_ids = {"error": str(e)}, None

    # ---- end to end through the C ABI with host buffers (pinned)
    last = ctx.download(G.F_LAST_ACC)["last_acc_mag"]
    h_pos = G.PinnedArray((3, n), np.float32)
    h_mass = G.PinnedArray((n,), np.float32)
    h_last = G.PinnedArray((n,), np.float32)
    h_acc = G.PinnedArray((3, n), np.float32)
    h_ids = G.PinnedArray((n,), np.uint32)
    h_oid = G.PinnedArray((n,), np.uint32)
    h_ids.array[:] = np.arange(n, dtype=np.uint32)
    h_pos.array[:] = p.pos.astype(np.float32)
    h_mass.array[:] = p.mass.astype(np.float32)
    h_last.array[ids.array] = last            # back to the host (input) order
    dist.barrier()
    ctx.timer_start()
    for _ in range(args.steps):
        # tvg_force_step_host: the copies overlap the keys, sort and walks
        ctx.force_step_host(n, h_pos.array, h_mass.array, last_acc=h_last.array, ids=h_ids.array,
                            grav_acc=h_acc.array, ids_out=h_oid.array, form=G.FORM_GROUP,
                            use_bh=False, parts=parts)
    e2e_ms = ctx.timer_stop()
    dist.barrier()
    t_e2e = dist.max(e2e_ms / args.steps) / 1e3
    e2e_value = dist.sum(n) / t_e2e
    h2d = n * 4 * 6        # pos[3], mass, last |a|, id
    d2h = n * 4 * 4        # grav_acc[3], id (the order of the result)

    # ---- roofline of the dominant kernel (the gravity walk)
    walk_flop = FLOP_PER_GRAV * (grav_i - quad_i) + FLOP_PER_QUAD * quad_i
    achieved = walk_flop / (walk_ms * 1e-3) / 1e12
    roofline = {
        "kernel": (f"k_walk_group<GM_CENTRE, {tune_choice}, float, "
                   f"{'monopole' if args.monopole else 'quadrupole'}> (gravity walk)"), "bound": "fp32",
        "achieved": round(achieved, 3), "peak": round(fp32_peak, 3), "unit": "TFLOP/s",
        "frac": round(achieved / fp32_peak, 4) if fp32_peak > 0 else None,
        "peak_source": "measured FFMA loop on this GPU (1.5 s, sustained under the power cap)",
        "traffic": None,
        "algorithmic": (f"{FLOP_PER_GRAV:.0f} flop x {(grav_i - quad_i) / args.steps / n:.0f} monopole"
                        f" + {FLOP_PER_QUAD:.0f} flop x {quad_i / args.steps / n:.0f} quadrupole"
                        " interactions/particle"),
    }
    prof = ROOT / "profiles" / "walk_group_traffic.json"
    if prof.exists():
        try:
            roofline["traffic"] = json.loads(prof.read_text()).get("bytes_per_launch_256")
        except (OSError, ValueError):
            pass

    # ---- the monopole group form (the reference's node moments) at its own
    # operating point, and at the plain form's opening parameter (the same
    # criterion as the plain form, on the same particles)
    monopole = matched = None
    if args.monopole:
        if not args.no_matched:
            matched = graph_steps(ctx, parts, args.steps, args.plain_open_rel, dist, n, G, tgt_ids)
            ctx.set_opening(0.25, args.open_rel)
    elif not args.no_monopole_run:
        cm, prep_err = None, None
        try:
            cm = G.GravityContext(n, float_bytes=4, periodic=True, boxsize=p.box,
                                  softening=p.softening, device=local)
            cm.upload(p.pos, p.mass)
            cm.set_domain((0.0, 0.0, 0.0), p.box)
            cm.ewald_init()
            cm.set_ewald_opening(MONO_OPEN[1])
            cm.force_step(form=G.FORM_GROUP, use_bh=True, parts=parts)
            cm.save_last_accel()
            cm.set_opening(0.25, MONO_OPEN[0])
            cm.force_step(form=G.FORM_GROUP, use_bh=False, parts=parts)
            if not args.tpl:
                cm.autotune(use_bh=False, parts=parts)
        except Exception as e:       # every rank still takes the collective steps below
            prep_err = str(e)
        try:
            monopole = graph_steps(cm, parts, min(args.steps, 2), MONO_OPEN[0], dist, n, G, tgt_ids,
                                   prep_err)
            if monopole.get("particles_per_s"):
                monopole["ewald_alpha"] = MONO_OPEN[1]
            if not args.no_matched:
                matched = graph_steps(cm, parts, args.steps, args.plain_open_rel, dist, n, G, tgt_ids,
                                      prep_err)
        finally:
            if cm is not None:
                cm.close()

    # ---- the same step with the learned Ewald correction: trained here by the
    # library's own kernels, validated against the exact table, then run in the walk
    learned = None
    if not args.no_mlp:
        ml_err = None
        try:
            ctx.timer_start()
            loss = ctx.mlp_train(steps=20000, batch=16384, n_samples=1 << 20, lr=2e-3, lr_final=1e-6,
                                 seed=3)
            train_ms = ctx.timer_stop()
            mx, rms = ctx.mlp_validate(max_allowed=1.0)
            for _ in range(3):                     # direct step, then the two captures
                ctx.step_graph(parts, G.EWALD_MLP)
            ml_ms = ml_ew = 0.0
            for _ in range(args.steps):
                ctx.timer_start()
                ctx.step_graph(parts, G.EWALD_MLP)
                ml_ms += ctx.timer_stop()
                ml_ew += ctx.phase_times()["ewald"]
        except Exception as e:       # every rank still takes the collective steps below
            ml_err, ml_ms = str(e), math.inf
        t_ml = dist.max(ml_ms / args.steps) / 1e3
        n_all = dist.sum(n)
    if not args.no_mlp and (ml_err is not None or not math.isfinite(t_ml)):
        learned = {"error": ml_err or "failed on another rank"}
    elif not args.no_mlp:
        learned = {"particles_per_s": n_all / t_ml, "ms_per_step": round(t_ml * 1e3, 2),
                   "ewald_walk_ms": round(ml_ew / args.steps, 2),
                   "train": {"steps": 20000, "batch": 16384, "samples": 1 << 20, "loss": loss,
                             "ms": round(train_ms, 1)},
                   "correction_error_vs_fp64_table": {"max": mx, "rms": rms},
                   "model": ("T = 4 pi x / 3 + seven nearest images + fitted cubic + s N(x); N "
                             "3-64-64-3 tanh, hidden layer on the tensor cores (mma.sync BF16, "
                             "FP32 accumulate, 32 points per warp); J and H from the Taylor table")}
        if tgt_ids is not None:
            try:
                ids_m = ctx.download(G.F_ID)["id"]
                inv = np.empty(n, np.int64)
                inv[ids_m] = np.arange(n)
                _, _, err_m = ctx.forcetest(np.sort(inv[tgt_ids]))
                learned["force_error"] = {k: float(f"{v:.4e}") for k, v in err_m.items()}
            except Exception as e:
                learned["force_error"] = {"error": str(e)}

    # ---- plain GPU form on a strided sample of active particles
    for a in (ids, h_pos, h_mass, h_last, h_acc, h_ids, h_oid):
        a.free()
    ctx.close()

    # ---- plain GPU form: the reference walk in FP64 (Float = double, exact
    # moments, table Ewald) on a strided sample of active particles
    plain = None
    if not args.no_plain:
        c64 = None
        try:
            c64 = G.GravityContext(n, float_bytes=8, periodic=True, boxsize=p.box,
                                   softening=p.softening, device=local)
            c64.upload(p.pos, p.mass)
            c64.set_domain((0.0, 0.0, 0.0), p.box)
            c64.ewald_init()
            c64.set_opening(0.25, args.plain_open_rel)
            c64.timer_start()
            c64.peano_keys()
            c64.sort_particles(want_perm=False)
            c64.top_nodes()
            c64.tree_build(exact_moments=True)
            pre_ms = c64.timer_stop()
            act = np.arange(0, n, args.plain_stride, dtype=np.int32)
            c64.set_active(act)
            c64.zero_accel()
            c64.walk(G.FORM_PLAIN, use_bh=True, parts=parts)      # prepare pass for |a_old|
            c64.save_last_accel()
            c64.timer_start()
            c64.walk(G.FORM_PLAIN, use_bh=False, parts=parts)
            w_ms = c64.timer_stop()
            g_pl, e_pl = c64.walk_counters()
            if tgt_ids is not None:
                # the same particles, walked in the plain form, against the same sum
                ids64 = c64.download(G.F_ID)["id"]
                inv = np.empty(n, np.int64)
                inv[ids64] = np.arange(n)
                t64 = np.sort(inv[tgt_ids])
                c64.set_active(t64.astype(np.int32))
                c64.zero_accel()
                c64.walk(G.FORM_PLAIN, use_bh=True, parts=parts)
                c64.save_last_accel()
                c64.zero_accel()
                c64.walk(G.FORM_PLAIN, use_bh=False, parts=parts)
                _, _, err64 = c64.forcetest(t64)
                accuracy["plain"] = {k: float(f"{v:.4e}") for k, v in err64.items()}
            t_plain = pre_ms * 1e-3 + w_ms * 1e-3 * n / len(act)
            plain = {"value": n / t_plain, "unit": UNIT,
                     "form": "plain: reference walk, one thread per particle, FP64, table Ewald",
                     "sample": ("keys, sort, build and the relative walk (incl. Ewald) of all "
                                f"{n} particles, measured" if args.plain_stride == 1 else
                                f"walk of every {args.plain_stride}th particle ({len(act)}), "
                                f"keys/sort/build for all, extrapolated"),
                     "ms_keys_sort_build": round(pre_ms, 2), "ms_walk_sample": round(w_ms, 2),
                     "interactions_per_particle": round((g_pl + e_pl) / len(act), 1),
                     "speedup_group_over_plain": round(value / ws / (n / t_plain), 2)}
            if matched and "particles_per_s" in matched:
                plain["speedup_group_over_plain_at_matched_opening"] = round(
                    matched["particles_per_s"] / ws / (n / t_plain), 2)
        except Exception as e:       # the headline line is printed all the same
            plain = {"error": str(e)}
        finally:
            if c64 is not None:
                c64.close()

    rungs = None
    if args.rung_steps > 0:
        try:
            rungs = rung_run(args, p, G, local)
        except Exception as e:
            rungs = {"error": str(e)}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
        try:
            cpu, err = cpu_reference(p, cores)
        except Exception as e:       # a failed or timed-out reference run
            cpu, err = None, str(e)
        if cpu is None:
            cpu = {"value": None, "unavailable": err}

    if rank == 0:
        ph = {k: round(statistics.mean(x[k] for x in phases), 3) for k in phases[0]}
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded Zel'dovich box, EH98 P(k), sigma8 0.8, n_s 0.96, z 50",
            "config": workload_config(args, p, ws),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": t_e2e * 1e3},
            "gpu_launches": int(launches),
            "clocks": clk,
            "phases_ms": ph,
            "interactions_per_particle": {"gravity": round(grav_i / args.steps / n, 1),
                                          "of_which_quadrupole": round(quad_i / args.steps / n, 1),
                                          "ewald_evaluations": round(ew_i / args.steps / n, 1)},
            "ewald_walk": {"kernel": f"k_ewald_group<{tune_choice}, false, float>",
                           "ms_per_step": round(ew_ms / args.steps, 2),
                           "evaluations_per_group": round(ew_i / args.steps / (n / (32 * tune_choice)), 1),
                           "evaluation": "Taylor-table K, dK, d2K: 15 float4 loads, ~200 FP32 ops"},
            "plain_form": plain,
            "group_form_monopole": monopole,
            "group_form_at_plain_opening": matched,
            "learned_ewald": learned,
            "device_memory_used_gb": hbm_gb,
            "accuracy": accuracy,
            "autotune": {"targets_per_lane": tune_choice,
                         "walk_ms_1_2_4_targets_per_lane": (None if tune_ms is None
                                                             else [round(x, 1) for x in tune_ms])},
            "rung_run": rungs,
        }
        print(json.dumps(out))
    dist.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
