"""Oracle for the hierarchical time integration: CPU restatement of the
reference's kick, drift, time-bin and timeline code in numpy.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path (tests/ import it).

FP32 (Float) and FP64 (double) arithmetic is replayed in the reference's
order with numpy scalars/arrays of the same width; numpy rounds every
operation (no fused multiply-add), as the CUDA file is compiled.

Parity pins:
* the kick/drift integrals against the Einstein-de Sitter closed forms
  (comoving.c:105-106: drift(a) = -2 / (H0 sqrt(a)), kick(a) = 2 sqrt(a) / H0)
  and against an adaptive quadrature (scipy.integrate.quad) for LCDM; the
  reference's own GSL QAG / cspline pair is not available here (GSL is not
  installed), so the spline itself is a restatement of the natural cubic
  spline the reference builds (comoving.c:146-150), knot 0 at a = 0
  (comoving.c:119: the table loop starts at i = 1);
* the per-particle updates (timestep.c:200-236, kick.c:9-70,
  drift.c:12-62, periodic.c:30-55) bit for bit.
"""
from __future__ import annotations

import math

import numpy as np

N_INT_BINS = 32
TABLESIZE = 512
FLT_MAX = float(np.finfo(np.float32).max)


def hubble(a, h0, om_m, om_l, om_r, om_0):
    """Hubble_Parameter / E_Hubble (cosmology.c:65-74)."""
    return h0 * math.sqrt(om_l + (1.0 - om_0) / (a * a) + om_m / (a * a * a) + om_r / (a ** 4))


def knots(time_begin, time_end):
    """Exp_Factor_Table (comoving.c:115-126): knot 0 stays at a = 0."""
    a0 = 0.95 * time_begin
    da = math.log((1.05 * time_end) / a0) / (TABLESIZE - 1)
    x = np.zeros(TABLESIZE)
    for i in range(1, TABLESIZE):
        x[i] = a0 * math.exp(da * i)
    return x, a0, da


def kd_integrals(time_begin, time_end, cosmo, quad=None):
    """Kick_Table / Drift_Table (comoving.c:119-137): int_{0.95 a_beg}^{a_i}
    da / (H a^2) and da / (H a^3); quad(f, lo, hi) integrates (default: scipy)."""
    if quad is None:
        from scipy.integrate import quad as sq

        def quad(f, lo, hi):
            return sq(f, lo, hi, epsabs=0.0, epsrel=1e-12, limit=200)[0]
    x, a0, _ = knots(time_begin, time_end)
    k = np.zeros(TABLESIZE)
    d = np.zeros(TABLESIZE)
    for i in range(1, TABLESIZE):
        k[i] = quad(lambda a: 1.0 / (hubble(a, *cosmo) * a * a), a0, x[i])
        d[i] = quad(lambda a: 1.0 / (hubble(a, *cosmo) * a * a * a), a0, x[i])
    return x, k, d


def natural_spline(x, y):
    """Second derivatives of the natural cubic spline through (x, y)."""
    n = len(x)
    m2 = np.zeros(n)
    cp = np.zeros(n)
    dp = np.zeros(n)
    for i in range(1, n - 1):
        hl, hr = x[i] - x[i - 1], x[i + 1] - x[i]
        r = 6.0 * ((y[i + 1] - y[i]) / hr - (y[i] - y[i - 1]) / hl)
        b = 2.0 * (hl + hr)
        if i == 1:
            cp[i], dp[i] = hr / b, r / b
        else:
            den = b - hl * cp[i - 1]
            cp[i], dp[i] = hr / den, (r - hl * dp[i - 1]) / den
    m2[n - 2] = dp[n - 2]
    for i in range(n - 3, 0, -1):
        m2[i] = dp[i] - cp[i] * m2[i + 1]
    return m2


def spline_eval(x, y, m2, a):
    i = int(np.searchsorted(x, a, side="right") - 1)
    i = max(0, min(i, len(x) - 2))
    h, d = x[i + 1] - x[i], a - x[i]
    b = (y[i + 1] - y[i]) / h - h * (2.0 * m2[i] + m2[i + 1]) / 6.0
    return y[i] + d * (b + d * (0.5 * m2[i] + d * (m2[i + 1] - m2[i]) / (6.0 * h)))


# ------------------------------------------------------------ particles

def timebins(grav_acc, bins, *, float_bytes, comoving, expansion_factor, hubble_parameter,
             time_int_accuracy, softening, step_max, dt_max_global, max_active_bin):
    """set_new_particle_timebins (timestep.c:200-236) with get_physical_timestep,
    cosmological_timestep (:496-527) and Acceleration_Physical (unit.c:55-71).
    Returns the new bins (int32)."""
    F = np.float32 if float_bytes == 4 else np.float64
    g = [np.asarray(grav_acc[k], dtype=F) for k in range(3)]
    a2 = (g[0] * g[0] + g[1] * g[1]) + g[2] * g[2]
    grav = np.sqrt(a2.astype(np.float64))
    if comoving:
        grav = grav * (1.0 / (expansion_factor * expansion_factor))
    acc_phys = grav.astype(F)
    eps = F(105.0 / 32.0 * softening)
    if comoving:
        dt_cosmo = (time_int_accuracy * np.sqrt(2 * expansion_factor * np.float64(eps)
                                                / acc_phys.astype(np.float64))).astype(np.float32)
    else:
        dt_cosmo = (time_int_accuracy * np.sqrt(2 * np.float64(eps)
                                                / acc_phys.astype(np.float64))).astype(np.float32)
    dtf = np.minimum(np.float64(FLT_MAX), dt_cosmo.astype(np.float64)).astype(np.float32)
    dt = dtf.astype(F)
    if comoving:
        dt = (dt.astype(np.float64) * hubble_parameter).astype(F)
    dt = np.minimum(dt.astype(np.float64), np.float64(np.float32(dt_max_global))).astype(F)
    _, e = np.frexp(step_max / dt.astype(np.float64))
    want = N_INT_BINS - 1 - e.astype(np.int64)
    allowed = np.maximum(max_active_bin, np.asarray(bins, np.int64))
    return np.minimum(want, allowed).astype(np.int32)


def kick(vel, acc, bins, it_kick, active, dt_of, float_bytes):
    """Kick_First_Halfstep / Kick_Second_Halfstep (kick.c:9-70) on copies;
    dt_of(it_curr, it_next) gives Particle_Kick_Step."""
    F = np.float32 if float_bytes == 4 else np.float64
    v = [np.array(vel[k], dtype=F) for k in range(3)]
    itk = np.array(it_kick, dtype=np.uint32)
    for i in active:
        step = np.uint32(1) << np.uint32(bins[i])
        c = itk[i]
        nx = np.uint32(c + (step >> np.uint32(1)))
        dt = F(dt_of(int(c), int(nx)))
        for k in range(3):
            v[k][i] = F(v[k][i] + F(dt * F(acc[k][i])))
        itk[i] = nx
    return v, itk


def drift(pos, vel, it_drift, active, it_next, dt_of, float_bytes):
    """Drift_To_Sync_Point (drift.c:12-40) on copies; dt_of gives
    Particle_Drift_Step."""
    F = np.float32 if float_bytes == 4 else np.float64
    x = [np.array(pos[k], dtype=F) for k in range(3)]
    itd = np.array(it_drift, dtype=np.uint32)
    for i in active:
        dt = np.float64(dt_of(int(itd[i]), int(it_next)))
        for k in range(3):
            x[k][i] = F(np.float64(x[k][i]) + dt * np.float64(vel[k][i]))
        itd[i] = np.uint32(it_next)
    return x, itd


def wrap(pos, box, float_bytes):
    """Periodic_Constrain_Particles_To_Box (periodic.c:30-55)."""
    F = np.float32 if float_bytes == 4 else np.float64
    out = []
    for k in range(3):
        v = np.array(pos[k], dtype=F)
        b = F(box)
        for i in range(len(v)):
            while v[i] < 0:
                v[i] = F(v[i] + b)
            while v[i] >= b:
                v[i] = F(v[i] - b)
        out.append(v)
    return out


def ctz(v):
    return (v & -v).bit_length() - 1


def system_step(st, time_bin_min, time_bin_max, it2time):
    """set_system_timestep + max_active_time_bin + the sync point test
    (timestep.c:44-69, 245-278) on a dict of the timeline state."""
    step_bin = 1 << time_bin_min
    step_sync = (1 << ctz(st["current"])) if st["current"] else 0
    if st["current"] == st["beg"]:
        step_sync = step_bin
    step_end = st["end"] - st["current"]
    st["step"] = min(step_end, step_bin, step_sync)
    st["next"] = st["current"] + st["step"]
    st["time_next"] = it2time(st["next"])
    st["time_step"] = st["time_next"] - st["time_current"]
    st["max_active_bin"] = ctz(st["next"])
    st["sync_point"] = 0
    if st["current"] == st["next_sync_point"]:
        st["sync_point"] = 1
        st["next_sync_point"] += 1 << time_bin_max
    return st
