"""Seeded synthetic initial conditions for the gravity hot path.

Two problem setups, restated from the formulas of the reference's own IC
generators (no code shared):

* ``hernquist`` -- isolated Hernquist (1990) halo, the setup of
  ``testing/Hernquist/src/make_ICs.pro:1-131``: radii by inverting the
  cumulative mass profile M(<r)/M = r^2/(r+a)^2 (truncated at 100 a), isotropic
  directions, speeds drawn by rejection from the isotropic distribution
  function f(E) of Hernquist (1990), eq. 17.
* ``zeldovich_box`` -- periodic cosmological box, the setup of
  ``testing/CosmoBox/src/make_ICs.pro:10-712``: a particle lattice displaced by
  the Zel'dovich approximation from a seeded Gaussian random field with the
  Eisenstein & Hu (1998) no-wiggle transfer function, normalised to sigma_8,
  scaled to the starting redshift with the linear growth factor.

Units follow the reference's code units (kpc/h, 1e10 Msun/h, km/s), in which
the gravitational constant is 43007.1 (``src/constants.c:5``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

# G in (kpc) (km/s)^2 / (1e10 Msun): GRAVITATIONAL_CONST / VELOCITY2CGS^2 *
# MASS2CGS / LENGTH2CGS with the reference's Config units (src/constants.c:5)
GRAVITY = 6.674e-8 / (1e5 ** 3) / (3.085677581e21 / 1e5) * 1.989e43


@dataclass
class Particles:
    """Structure-of-arrays particle set (float64 on the host)."""

    pos: np.ndarray        # (3, n)
    vel: np.ndarray        # (3, n)
    mass: np.ndarray       # (n,)
    box: float             # periodic box size, 0 for isolated
    softening: float       # Plummer-equivalent softening length
    a_start: float = 1.0   # expansion factor (1 when not cosmological)

    @property
    def n(self) -> int:
        return int(self.mass.shape[0])


# ---------------------------------------------------------------- Hernquist

def _hernquist_df(E: np.ndarray, G: float, M: float, a: float) -> np.ndarray:
    """Isotropic Hernquist distribution function f(E), E < 0 (Hernquist 1990)."""
    vg = math.sqrt(G * M / a)
    q = np.sqrt(np.clip(-E * a / (G * M), 0.0, 1.0 - 1e-15))
    q2 = q * q
    pref = M / (8.0 * math.sqrt(2.0) * math.pi ** 3 * a ** 3 * vg ** 3)
    body = (3.0 * np.arcsin(q) + q * np.sqrt(1.0 - q2) * (1.0 - 2.0 * q2)
            * (8.0 * q2 * q2 - 8.0 * q2 - 3.0))
    return pref * body / (1.0 - q2) ** 2.5


def hernquist(n: int = 65536, seed: int = 42, a: float = 1.0, mass: float = 1.0,
              r_trunc: float = 100.0, softening: float = 0.01,
              G: float = GRAVITY) -> Particles:
    """Isolated Hernquist halo of ``n`` equal-mass particles (seeded)."""
    rng = np.random.default_rng(seed)
    qmax = (r_trunc / (1.0 + r_trunc)) ** 2
    q = rng.uniform(0.0, qmax, n)
    sq = np.sqrt(q)
    r = a * sq / (1.0 - sq)
    cost = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * math.pi, n)
    sint = np.sqrt(1.0 - cost * cost)
    pos = np.stack([r * sint * np.cos(phi), r * sint * np.sin(phi), r * cost])

    # speeds: p(v | r) ~ v^2 f(Phi(r) + v^2/2) on [0, v_esc]
    pot = -G * mass / (r + a)
    vesc = np.sqrt(-2.0 * pot)
    speed = np.empty(n)
    todo = np.arange(n)
    # envelope from a per-particle grid maximum
    grid = np.linspace(0.0, 1.0, 64)[1:-1]
    fmax = np.zeros(n)
    for x in grid:
        v = x * vesc
        fmax = np.maximum(fmax, v * v * _hernquist_df(pot + 0.5 * v * v, G, mass, a))
    fmax *= 1.2
    while todo.size:
        v = rng.uniform(0.0, 1.0, todo.size) * vesc[todo]
        u = rng.uniform(0.0, 1.0, todo.size) * fmax[todo]
        f = v * v * _hernquist_df(pot[todo] + 0.5 * v * v, G, mass, a)
        ok = u <= f
        speed[todo[ok]] = v[ok]
        todo = todo[~ok]
    cost = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * math.pi, n)
    sint = np.sqrt(1.0 - cost * cost)
    vel = np.stack([speed * sint * np.cos(phi), speed * sint * np.sin(phi), speed * cost])
    m = np.full(n, mass / n)
    return Particles(pos=pos, vel=vel, mass=m, box=0.0, softening=softening)


# ------------------------------------------------------------ cosmology box

@dataclass
class Cosmology:
    omega_m: float = 0.3
    omega_l: float = 0.7
    omega_b: float = 0.04
    h: float = 0.7
    sigma8: float = 0.8
    n_s: float = 0.96
    t_cmb: float = 2.725

    def E(self, a):
        ok = 1.0 - self.omega_m - self.omega_l
        return np.sqrt(self.omega_m / a ** 3 + ok / a ** 2 + self.omega_l)

    def transfer_eh_nowiggle(self, k_h):
        """Eisenstein & Hu (1998) zero-baryon-wiggle transfer function, k in h/Mpc."""
        om, ob, h = self.omega_m, self.omega_b, self.h
        theta = self.t_cmb / 2.7
        omh2, obh2 = om * h * h, ob * h * h
        fb = ob / om
        s = 44.5 * math.log(9.83 / omh2) / math.sqrt(1.0 + 10.0 * obh2 ** 0.75)
        alpha = 1.0 - 0.328 * math.log(431.0 * omh2) * fb + 0.38 * math.log(22.3 * omh2) * fb * fb
        k_mpc = k_h * h
        gamma = om * h * (alpha + (1.0 - alpha) / (1.0 + (0.43 * k_mpc * s) ** 4))
        q = k_h * theta * theta / gamma
        L0 = np.log(2.0 * math.e + 1.8 * q)
        C0 = 14.2 + 731.0 / (1.0 + 62.5 * q)
        return L0 / (L0 + C0 * q * q)

    def growth(self, a: float) -> float:
        """Linear growth factor D(a), normalised to D(1)=1 (integral form)."""
        def unnorm(aa):
            x = np.linspace(1e-6, aa, 20001)
            integrand = 1.0 / (x * self.E(x)) ** 3
            integ = np.trapezoid(integrand, x)
            return 2.5 * self.omega_m * self.E(aa) * integ
        return unnorm(a) / unnorm(1.0)

    def growth_rate(self, a: float) -> float:
        da = 1e-4 * a
        return (math.log(self.growth(a + da)) - math.log(self.growth(a - da))) / (
            math.log(a + da) - math.log(a - da))

    def power_norm(self) -> float:
        """Amplitude A so that A k^n_s T^2(k) has sigma(8 Mpc/h) = sigma_8 at a=1."""
        k = np.logspace(-5, 3, 200001)
        x = 8.0 * k
        w = 3.0 * (np.sin(x) - x * np.cos(x)) / x ** 3
        p = k ** self.n_s * self.transfer_eh_nowiggle(k) ** 2
        s2 = np.trapezoid(k * k * p * w * w, k) / (2.0 * math.pi ** 2)
        return self.sigma8 ** 2 / s2


def zeldovich_box(n_side: int = 128, box_mpc: float = 100.0, z_start: float = 50.0,
                  seed: int = 1234, cosmo: Cosmology | None = None,
                  softening_frac: float = 1.0 / 30.0) -> Particles:
    """Lattice of ``n_side^3`` particles with Zel'dovich displacements (seeded).

    Lengths in kpc/h, box ``box_mpc`` Mpc/h, velocities are the reference's
    internal comoving variable a^2 dx/dt (km/s), masses in 1e10 Msun/h.
    """
    cosmo = cosmo or Cosmology()
    L = box_mpc * 1000.0
    n = n_side
    a = 1.0 / (1.0 + z_start)
    amp = cosmo.power_norm()
    dgrow = cosmo.growth(a)
    frate = cosmo.growth_rate(a)

    rng = np.random.default_rng(seed)
    white = rng.standard_normal((n, n, n)).astype(np.float64)
    wk = np.fft.rfftn(white)
    del white
    kf = 2.0 * math.pi / box_mpc                      # h/Mpc
    k1 = np.fft.fftfreq(n, d=1.0 / n) * kf
    kz = np.fft.rfftfreq(n, d=1.0 / n) * kf
    kx = k1[:, None, None]
    ky = k1[None, :, None]
    kzz = kz[None, None, :]
    k2 = kx * kx + ky * ky + kzz * kzz
    k2[0, 0, 0] = 1.0
    kmag = np.sqrt(k2)
    pk = amp * kmag ** cosmo.n_s * cosmo.transfer_eh_nowiggle(kmag) ** 2   # (Mpc/h)^3
    vol = box_mpc ** 3
    scale = np.sqrt(pk / vol) * math.sqrt(n ** 3) * dgrow
    knyq = kf * n / 2
    scale[kmag > knyq] = 0.0
    scale[0, 0, 0] = 0.0
    delta_k = wk * scale
    del wk, scale, pk
    disp = np.empty((3, n, n, n))
    for d, kc in enumerate((kx, ky, kzz)):
        # psi_k = i k / k^2 delta_k  (Mpc/h); displacement in kpc/h
        disp[d] = np.fft.irfftn(1j * kc / k2 * delta_k, s=(n, n, n), axes=(0, 1, 2)) * 1000.0
    del delta_k
    spacing = L / n
    g = (np.arange(n) + 0.5) * spacing
    qx, qy, qz = np.meshgrid(g, g, g, indexing="ij")
    pos = np.stack([qx, qy, qz]).reshape(3, -1) + disp.reshape(3, -1)
    pos = inside_box(np.mod(pos, L), L)
    # peculiar velocity a*H*f*D-scaled displacement; internal variable a^2 dx/dt
    hub = 0.1 * cosmo.E(a)                           # km/s per kpc/h
    vel = disp.reshape(3, -1) * (a * hub * frate) * a
    rho_crit = 3.0 * 0.1 ** 2 / (8.0 * math.pi * GRAVITY)
    mpart = cosmo.omega_m * rho_crit * L ** 3 / n ** 3
    mass = np.full(n ** 3, mpart)
    return Particles(pos=pos, vel=vel, mass=mass, box=L,
                     softening=spacing * softening_frac, a_start=a)


def inside_box(pos: np.ndarray, box: float) -> np.ndarray:
    """Positions in [0, box) in float64 and in float32 alike. np.mod can return
    box itself for tiny negative inputs, and a float64 position just below the
    box can round up to box in float32; such coordinates become the largest
    float32 below box. The reference wraps positions into the box before its
    first keys (Periodic_Constrain_Particles_To_Box, periodic.c:30-55): a
    coordinate equal to the box would otherwise take the key of coordinate 0
    and break the tree's PH contiguity."""
    below = float(np.nextafter(np.float32(box), np.float32(0.0)))
    return np.where(pos.astype(np.float32) >= np.float32(box), below, pos)


def random_box(n: int, box: float = 1000.0, seed: int = 7, clumps: int = 0) -> Particles:
    """Uniform random periodic box (optionally with Gaussian clumps), for tests."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0.0, box, (3, n))
    if clumps:
        m = n // 4
        centres = rng.uniform(0.0, box, (3, clumps))
        which = rng.integers(0, clumps, m)
        pos[:, :m] = np.mod(centres[:, which] + rng.normal(0.0, 0.02 * box, (3, m)), box)
    pos = inside_box(pos, box)
    vel = rng.normal(0.0, 1.0, (3, n))
    mass = np.full(n, 1.0 / n)
    return Particles(pos=pos, vel=vel, mass=mass, box=box,
                     softening=box / n ** (1.0 / 3.0) / 30.0)
