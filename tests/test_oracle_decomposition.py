"""The restatement of Domain_Decomposition's cost-balanced top nodes
(oracle/decomposition.py) against the reference itself.

The fixtures (tests/golden/decomp_*.npz, made by `make_golden.py
decomposition`) hold the reference's second decomposition -- the one that
balances the P.Cost left by a first force computation over NTask = 3 or 8
OpenMP threads (domain.c:67-145, 151-156) -- with its tree and both walks.
The restatement must reproduce the top nodes (key, level, first particle,
count, order) exactly; the oracle pipeline on those top nodes must reproduce
the tree, Tree_Parent and the Barnes-Hut pass bit for bit.
"""
import numpy as np
import pytest

import decomposition
from pipeline import oracle_pipeline, oracle_ewald_tables, assert_struct_equal

CASES = ["decomp_hernquist_iso_f64_t3", "decomp_clumpy_per_f32_t8"]
TREE_FIELDS = ["DNext", "Bitfield", "DUp", "Npart", "Pos", "Mass", "CoM"]
TOP_FIELDS = ["Key", "Target", "Level", "First_Part", "Npart", "Pos", "Mass", "CoM"]


def cost_by_input_index(g):
    """P.Cost before the second decomposition, indexed by particle ID (= input index)."""
    c = np.empty(len(g["cost_in"]))
    c[g["id_in"].astype(np.int64)] = g["cost_in"]
    return c


@pytest.mark.parametrize("case", CASES)
def test_restated_top_nodes_equal_the_reference(golden_dir, case):
    g = np.load(golden_dir / f"{case}.npz")
    top = g["topnodes"]
    cost_sorted = cost_by_input_index(g)[g["perm"].astype(np.int64)]
    bunches, rounds = decomposition.decompose(g["std_key"][:, 0], cost_sorted, int(g["ntask"]))
    assert rounds > 0                      # the balanced case, not the level-2 cells
    assert len(bunches) == len(top)
    got = np.array([(k, lv, f, n) for k, lv, f, n in bunches], dtype=np.uint64)
    assert np.array_equal(got[:, 0], top["Key"])
    assert np.array_equal(got[:, 1].astype(np.int64), top["Level"])
    assert np.array_equal(got[:, 2].astype(np.int64), top["First_Part"])
    assert np.array_equal(got[:, 3].astype(np.int64), top["Npart"])
    assert len(np.unique(top["Level"])) > 1


@pytest.mark.parametrize("case", CASES)
def test_oracle_pipeline_on_balanced_top_nodes(golden_dir, case):
    g = np.load(golden_dir / f"{case}.npz")
    fsize, box = int(g["float_size"]), float(g["box"])
    ew = oracle_ewald_tables(fsize, box) if box > 0 else None
    o = oracle_pipeline(g["pos_in"], g["mass_in"], g["domain_origin"], float(g["domain_size"][0]),
                        fsize, box=box, softening=float(g["softening"]), gravity=float(g["gravity"][0]),
                        ewald=ew, passes=("bh",), ntask=int(g["ntask"]), cost=cost_by_input_index(g))
    assert np.array_equal(o["perm"], g["perm"])
    assert_struct_equal(o["top"], g["topnodes"], TOP_FIELDS, "topnodes")
    assert_struct_equal(o["tree"], g["tree"], TREE_FIELDS, "tree")
    assert np.array_equal(o["tree_parent"], g["tree_parent"])
    assert np.array_equal(o["bh_cost"].astype(np.float64), g["bh_cost"])
    assert np.array_equal(o["bh_gacc"].astype(np.float64), g["bh_gacc"])
