"""Writes tvg_uniform_cube.inc: the polynomial that the group form's Ewald
walk (tvg_walk_group.cu, uniform_remainder) uses for the field of the
uniform background beyond its linear term.

The field of the uniform unit-density cube [-1/2, 1/2]^3 at tau (G = 1) has
a closed form: over the cube's corners, the double antiderivative of 1/r of
a rectangular prism, F = Y ln(Z + r) + Z ln(Y + r) - X atan(Y Z / (X r))
(Nagy 1966). Near the centre g(tau) = -4 pi tau / 3 + O(tau^3), and the
remainder R_x(tau) = g_x(tau) + 4 pi tau_x / 3 is an odd polynomial series
with the cube's symmetry: odd in tau_x, even and symmetric in tau_y and
tau_z. The walk expands about the group centre only for groups narrower than
a twentieth of the box, so |tau_i| < 0.05. A least-squares fit of the
degree-7 terms on a 24^3 Chebyshev grid of [-0.06, 0.06]^3 matches the closed
form within 2e-8 of max |R| there; the closed form in FP64 costs 24
logarithm pairs and arctangents per particle.

Run: python tandav_b200/csrc/gen_uniform_cube.py (rewrites the .inc beside it).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

HALF = 0.06          # fitted half-width (box units)
GRID = 24            # Chebyshev points per axis
DEGREES = (3, 5, 7)


def prism_f(X, Y, Z):
    r = np.sqrt(X * X + Y * Y + Z * Z)
    return Y * np.log(Z + r) + Z * np.log(Y + r) - X * np.arctan(Y * Z / (X * r))


def cube_field_x(x, y, z):
    """x component of the unit cube's field at (x, y, z), closed form."""
    a1, a2, b1, b2, c1, c2 = -0.5 - x, 0.5 - x, -0.5 - y, 0.5 - y, -0.5 - z, 0.5 - z
    return ((prism_f(a1, b2, c2) - prism_f(a2, b2, c2)) - (prism_f(a1, b1, c2) - prism_f(a2, b1, c2))
            - (prism_f(a1, b2, c1) - prism_f(a2, b2, c1)) + (prism_f(a1, b1, c1) - prism_f(a2, b1, c1)))


def remainder_x(x, y, z):
    return cube_field_x(x, y, z) + 4.0 * np.pi / 3.0 * x


def terms():
    """(a, b, c) exponents: x^a (y^b z^c + y^c z^b), b <= c (one term if b == c)."""
    out = []
    for d in DEGREES:
        for a in range(1, d + 1, 2):
            rest = d - a
            for b in range(0, rest + 1, 2):
                c = rest - b
                if b <= c:
                    out.append((a, b, c))
    return out


def basis(x, y, z):
    cols = []
    for a, b, c in terms():
        sym = y ** b * z ** c if b == c else y ** b * z ** c + y ** c * z ** b
        cols.append(x ** a * sym)
    return np.stack(cols, 1)


def fit():
    k = np.arange(GRID)
    u = HALF * np.cos(np.pi * (k + 0.5) / GRID)
    x, y, z = (g.ravel() for g in np.meshgrid(u, u, u, indexing="ij"))
    A = basis(x, y, z)
    scale = HALF ** -np.array([a + b + c for a, b, c in terms()], dtype=np.float64)
    coef, *_ = np.linalg.lstsq(A * scale, remainder_x(x, y, z), rcond=None)
    return coef * scale


def evaluate(coef, x, y, z):
    """The .inc's polynomial for the x component, FP64."""
    return basis(np.asarray(x, np.float64), np.asarray(y, np.float64), np.asarray(z, np.float64)) @ coef


def render(coef) -> str:
    names = [f"x^{a} (y^{b} z^{c}" + (")" if b == c else f" + y^{c} z^{b})") for a, b, c in terms()]
    lines = ["// Written by gen_uniform_cube.py (do not edit): the field of the uniform",
             "// unit-density cube beyond its linear term, R_x = g_x + 4 pi x / 3, near its",
             "// centre, as sum_k kUniformCube[k] * term_k:"]
    lines += [f"//   {i:2d}: {n}" for i, n in enumerate(names)]
    lines.append(f"constexpr int kUniformCubeTerms = {len(coef)};")
    lines.append("constexpr double kUniformCube[kUniformCubeTerms] = {")
    lines += [f"\t{float(c)!r}," for c in coef]
    lines.append("};")
    return "\n".join(lines) + "\n"


def main():
    out = Path(__file__).resolve().parent / "tvg_uniform_cube.inc"
    out.write_text(render(fit()))
    print(f"wrote {out}")


if __name__ == "__main__":
    main()
