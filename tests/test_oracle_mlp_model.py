"""The learned Ewald correction's model (oracle restatement in
oracle/mlp.py): what the network is left to learn. After the background term
4 pi x / 3 and the seven lattice images nearest to the octant, a
least-squares cubic in v = 4 x - 1 leaves ~1.6e-3 rms of T (|T| up to ~4).
Without the images the same cubic leaves over ten times more; the steep part
near the faces and corners is what the images carry. FP64 lattice sums from
the oracle's restatement of compute_ewald_force (Gravity/periodic.c:352-461)."""
import numpy as np

import mlp as O
import port


def _cubic_residual(x, r):
    m = O.monomials(4.0 * x - 1.0)
    coef, *_ = np.linalg.lstsq(m, r, rcond=None)
    return r - m @ coef


def test_cubic_fit_after_images_leaves_a_small_rest():
    rng = np.random.default_rng(5)
    x = rng.uniform(0.0, 0.5, (8192, 3))
    t = port.ewald_force(x)
    rest = _cubic_residual(x, t - O.analytic(x))
    rms = np.sqrt((rest ** 2).mean())
    assert rms < 2.5e-3 and np.abs(rest).max() < 1.5e-2
    # the background term alone: the cubic cannot follow the images
    rest0 = _cubic_residual(x, t - O.LIN * x)
    assert np.sqrt((rest0 ** 2).mean()) > 10 * rms
