"""The uniform-background remainder of the group form's Ewald expansion
(tvg_walk_group.cu, uniform_remainder): the polynomial in
tandav_b200/csrc/tvg_uniform_cube.inc against the closed form of the uniform
cube's field that gen_uniform_cube.py fits it to, and that closed form
against the properties it must have. No reference counterpart (the
reference's Ewald walk has no expansion about a group centre)."""
import re
import sys
from pathlib import Path

import numpy as np

CSRC = Path(__file__).resolve().parents[1] / "tandav_b200" / "csrc"
sys.path.insert(0, str(CSRC))
import gen_uniform_cube as guc  # noqa: E402


def committed_coefficients():
    text = (CSRC / "tvg_uniform_cube.inc").read_text()
    body = text[text.index("kUniformCube[kUniformCubeTerms] = {"):]
    return np.array([float(v) for v in re.findall(r"^\t(\S+),$", body, re.M)])


def field(x, y, z):
    """The cube's field (all three components) from the closed form."""
    return np.stack([guc.cube_field_x(x, y, z), guc.cube_field_x(y, x, z), guc.cube_field_x(z, x, y)])


def test_closed_form_properties():
    rng = np.random.default_rng(7)
    # odd, with the cube's symmetry: g_x(x, y, z) = g_x(x, z, y) = g_x(x, -y, z)
    x, y, z = rng.uniform(-0.3, 0.3, (3, 200))
    gx = guc.cube_field_x(x, y, z)
    np.testing.assert_allclose(guc.cube_field_x(-x, y, z), -gx, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(guc.cube_field_x(x, z, y), gx, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(guc.cube_field_x(x, -y, z), gx, rtol=1e-12, atol=1e-14)
    # inside: div g = -4 pi (unit density), so near the centre g = -4 pi tau / 3
    t = np.array([1e-4, -2e-4, 3e-4])
    np.testing.assert_allclose(field(*t), -4 * np.pi / 3 * t, rtol=1e-6)
    h = 1e-4
    for p in rng.uniform(-0.4, 0.4, (5, 3)):
        div = sum((field(*(p + h * e))[k] - field(*(p - h * e))[k]) / (2 * h)
                  for k, e in enumerate(np.eye(3)))
        assert abs(div + 4 * np.pi) < 1e-5
    # far away: a unit point mass (the cube's quadrupole vanishes)
    p = np.array([6.0, 1.5, -3.0])
    np.testing.assert_allclose(field(*p), -p / np.linalg.norm(p) ** 3, rtol=2e-4)


def test_committed_polynomial_matches_the_closed_form():
    coef = committed_coefficients()
    assert len(coef) == len(guc.terms())
    rng = np.random.default_rng(11)
    x, y, z = rng.uniform(-0.05, 0.05, (3, 100000))
    r = guc.remainder_x(x, y, z)
    err = np.abs(guc.evaluate(coef, x, y, z) - r).max()
    assert err < 5e-8 * np.abs(r).max(), err
    # the committed table is the generator's current fit
    np.testing.assert_allclose(coef, guc.fit(), rtol=1e-8, atol=1e-10)
    # the walk evaluates y and z by permuting the arguments
    ry = guc.cube_field_x(y, x, z) + 4 * np.pi / 3 * y
    assert np.abs(guc.evaluate(coef, y, x, z) - ry).max() < 5e-8 * np.abs(ry).max()
