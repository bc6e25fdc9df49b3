"""Generates the golden fixtures in tests/golden/ by running the REAL reference.

The reference C sources are compiled unmodified by `make -C oracle ref` into
oracle/_ref/<variant>/ref_harness; this script feeds them seeded inputs and
stores their outputs (keys, sort permutation, top nodes, tree, Tree_Parent,
accelerations of the BH and relative passes, Ewald parts) as compressed .npz
files. Re-run after changing the inputs: `python tests/golden/make_golden.py`
(`... make_golden.py potential` for the potential fixtures only,
`... make_golden.py decomposition` for the balanced decompositions only,
`... make_golden.py vector_size` for the smaller-VECTOR_SIZE builds only).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

import refrun  # noqa: E402
from tandav_b200 import ics  # noqa: E402


def keys_case():
    """Test_Peanokey's 4^3 grid (peano.c:344-361), the 1-1e-10 corner
    (peano.c:323-325), cube corners and seeded random points, unit box."""
    pts = []
    n, delta = 4, 0.25
    for i in range(n):
        for j in range(n):
            for k in range(n):
                pts.append(((i + 0.5) * delta, (j + 0.5) * delta, (k + 0.5) * delta))
    pts.append((0.9999999999,) * 3)
    for c in range(8):
        pts.append(tuple(0.0 if not (c >> b) & 1 else 1.0 - 2.0 ** -30 for b in range(3)))
    rng = np.random.default_rng(11)
    pts.extend(map(tuple, rng.uniform(0, 1, (200, 3))))
    pos = np.array(pts).T.copy()
    out = {"pos": pos}
    for variant in ("iso_f32", "iso_f64"):
        r = refrun.run(variant, "keys", pos, origin=(0.0, 0.0, 0.0), size=1.0)
        out[f"{variant}_std"] = r["std_key"]
        out[f"{variant}_rev"] = r["rev_key"]
    np.savez_compressed(HERE / "keys_grid.npz", **out)


def force_case(name, variant, p, flags=3, vector_size=64):
    r = refrun.run(variant, "force", p.pos, p.vel, p.mass, box=p.box, softening=p.softening,
                   flags=flags)
    out = dict(pos_in=p.pos, mass_in=p.mass, box=np.array(p.box), softening=np.array(p.softening),
               vector_size=np.array(vector_size),
               float_size=np.array(r["float_size"]), gravity=r["gravity"],
               domain_size=r["domain_size"], domain_origin=r["domain_origin"],
               perm=r["perm"], std_key=r["std_key"], rev_key=r["rev_key"],
               topnodes=r["topnodes"], tree=r["tree"], tree_parent=r["tree_parent"],
               last_acc_mag=r["last_acc_mag"])
    for part in ("bh", "rel", "bhew", "relew"):
        for q in ("gacc", "acc", "cost", "pot"):
            k = f"{part}_{q}"
            if k in r:
                out[k] = r[k]
    np.savez_compressed(HERE / f"{name}.npz", **out)


def decomposition_case(name, variant, p, ntask):
    """The reference's second Domain_Decomposition (mode force2) at `ntask`
    OpenMP threads: top nodes balanced by the P.Cost of a first force
    computation, the tree and both passes on them."""
    r = refrun.run(variant, "force2", p.pos, p.vel, p.mass, box=p.box, softening=p.softening,
                   flags=3, threads=ntask)
    out = dict(pos_in=p.pos, mass_in=p.mass, box=np.array(p.box), softening=np.array(p.softening),
               ntask=np.array(ntask), float_size=np.array(r["float_size"]), gravity=r["gravity"],
               domain_size=r["domain_size"], domain_origin=r["domain_origin"],
               cost_in=r["cost_in"], id_in=r["id_in"], perm=r["perm"], std_key=r["std_key"],
               rev_key=r["rev_key"], topnodes=r["topnodes"], tree=r["tree"],
               tree_parent=r["tree_parent"], last_acc_mag=r["last_acc_mag"])
    for part in ("bh", "rel", "bhew", "relew"):
        for q in ("gacc", "cost"):
            k = f"{part}_{q}"
            if k in r:
                out[k] = r[k]
    np.savez_compressed(HERE / f"{name}.npz", **out)


def decomposition_cases():
    decomposition_case("decomp_hernquist_iso_f64_t3", "iso_f64", ics.hernquist(n=16384, seed=43), 3)
    decomposition_case("decomp_clumpy_per_f32_t8", "per_f32",
                       ics.random_box(20000, box=1000.0, seed=44, clumps=5), 8)


def main():
    keys_case()
    force_case("hernquist_iso_f64", "iso_f64", ics.hernquist(n=2048, seed=5))
    force_case("hernquist_iso_f32", "iso_f32", ics.hernquist(n=2048, seed=6))
    force_case("box_per_f32", "per_f32", ics.random_box(3000, box=1000.0, seed=8, clumps=6))
    force_case("zeldovich_per_f64", "per_f64", ics.zeldovich_box(n_side=20, seed=9))


def vector_size_cases():
    """The reference built with a smaller VECTOR_SIZE (variants *_v<N>)."""
    force_case("box_per_f32_v32", "per_f32_v32",
               ics.random_box(3000, box=1000.0, seed=8, clumps=6), vector_size=32)
    force_case("hernquist_iso_f64_v16", "iso_f64_v16", ics.hernquist(n=2048, seed=5),
               vector_size=16)


def potential_cases():
    """The same inputs through the reference built with GRAVITY_POTENTIAL
    (variants *_pot): forces and Grav_Pot of both passes."""
    force_case("hernquist_iso_f64_pot", "iso_f64_pot", ics.hernquist(n=2048, seed=5))
    force_case("hernquist_iso_f32_pot", "iso_f32_pot", ics.hernquist(n=2048, seed=6))
    force_case("zeldovich_per_f64_pot", "per_f64_pot", ics.zeldovich_box(n_side=20, seed=9))


if __name__ == "__main__":
    # `make_golden.py potential` writes only the potential fixtures
    if sys.argv[1:] == ["potential"]:
        potential_cases()
    elif sys.argv[1:] == ["decomposition"]:
        decomposition_cases()
    elif sys.argv[1:] == ["vector_size"]:
        vector_size_cases()
    else:
        main()
