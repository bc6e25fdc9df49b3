"""The Taylor-table scheme of the group form's Ewald walk (oracle
restatement in oracle/ewald_taylor.py) against direct lattice sums at
points between the nodes: the value to 4e-7 of |T| and the gradient to 3e-5
of its largest component with 33 nodes per axis, at nodes near the origin,
the face centres, the edges and the corner of the octant."""
import numpy as np
import pytest

import ewald_taylor as TT
import port

N = 33
G = 2 * (N - 1)
NODES = [(0, 0, 0), (1, 1, 1), (32, 0, 0), (31, 1, 0), (16, 10, 3), (32, 16, 0), (20, 32, 5),
         (32, 32, 0), (32, 32, 32)]


@pytest.mark.parametrize("node", NODES)
def test_taylor_record_against_lattice_sums(node):
    rec = TT.record(node, N)
    rng = np.random.default_rng(sum(node) + 7)
    for _ in range(4):
        # offsets the lookup can meet: |du| <= 1/2, and du >= 0 on the
        # octant's lower faces
        du = rng.uniform(-0.5, 0.5, 3)
        du = np.where(np.asarray(node) == 0, np.abs(du), du)
        x = (np.asarray(node) + du) / G
        val, grad, _ = TT.evaluate(rec, du)
        exact = port.ewald_force(x)[0]
        assert np.abs(val - exact).max() <= 4e-7 * max(np.linalg.norm(exact), 1e-2)
        e = 1e-4
        jac = np.zeros((3, 3))
        for b in range(3):
            xp, xm = x.copy(), x.copy()
            xp[b] += e / G
            xm[b] -= e / G
            jac[:, b] = (port.ewald_force(xp)[0] - port.ewald_force(xm)[0]) / (2 * e)
        assert np.abs(grad - jac).max() <= 3e-5 * max(np.abs(jac).max(), 1e-3)
