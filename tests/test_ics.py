"""Seeded initial conditions: determinism and the physical properties they
are defined by."""
import math

import numpy as np

from tandav_b200 import ics


def test_hernquist_profile_and_seed():
    a = ics.hernquist(n=20000, seed=3)
    b = ics.hernquist(n=20000, seed=3)
    assert np.array_equal(a.pos, b.pos) and np.array_equal(a.vel, b.vel)
    r = np.sqrt((a.pos ** 2).sum(0))
    # M(<r) = r^2/(1+r)^2 (truncated at 100 a): half of the truncated mass at
    # r_h with r_h^2/(1+r_h)^2 = 0.5 * (100/101)^2
    q = math.sqrt(0.5) * 100 / 101
    r_half = q / (1 - q)
    assert abs(np.median(r) - r_half) / r_half < 0.03
    assert r.max() <= 100.0 + 1e-9
    # bound orbits: speed below escape speed
    v = np.sqrt((a.vel ** 2).sum(0))
    vesc = np.sqrt(2 * ics.GRAVITY / (r + 1))
    assert np.all(v <= vesc * (1 + 1e-12))
    assert abs(a.mass.sum() - 1.0) < 1e-12


def test_zeldovich_box_properties():
    p = ics.zeldovich_box(n_side=16, seed=1)
    L = 100000.0
    assert p.pos.shape == (3, 16 ** 3)
    assert p.pos.min() >= 0 and p.pos.max() < L
    assert abs(p.softening - L / 16 / 30) < 1e-9
    # displacements small against the mean spacing at z = 50
    g = (np.arange(16) + 0.5) * L / 16
    q = np.stack(np.meshgrid(g, g, g, indexing="ij")).reshape(3, -1)
    d = (p.pos - q + L / 2) % L - L / 2
    assert 0 < np.sqrt((d ** 2).mean()) < 0.5 * L / 16
    # total mass = Omega_m rho_crit L^3
    rho_crit = 3 * 0.01 / (8 * math.pi * ics.GRAVITY)
    assert abs(p.mass.sum() / (0.3 * rho_crit * L ** 3) - 1) < 1e-12
    q2 = ics.zeldovich_box(n_side=16, seed=1)
    assert np.array_equal(p.pos, q2.pos)
