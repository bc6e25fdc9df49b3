"""The tree updates between rebuilds (src/Gravity/tree_update.c) in the
restatement (oracle/tree_update.py) against the reference itself: the
harness's mode "update" runs Gravity_Tree_Update_Kicks for two kick passes
over a subset of the particles and Gravity_Tree_Update_Drift on the tree it
has just built, then both walks on the updated tree. Every tree and top-node
field after the kicks (Dp, the UPDATED bits, negative top-node levels) and
after the drift (CoM), and the accelerations of the walks on the updated
tree (port.walk), must agree bit for bit. The library's own per-node
functions (tandav_b200/csrc/tvg_tree_update.cuh, built for the host by
tests/tree_update_host.cu) are held against the same reference output."""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import port
import refrun
import tree_update as TU
from pipeline import assert_struct_equal, oracle_ewald_tables
from tandav_b200 import ics

TREE_FIELDS = ("DNext", "Bitfield", "DUp", "Npart", "Pos", "Mass", "CoM", "Dp")
TOP_FIELDS = ("Key", "Target", "Level", "First_Part", "Npart", "Pos", "Mass", "CoM", "Dp")
KICK_DT, DRIFT_DT = 0.004, 0.5

CASES = [("iso_f32", "hernquist"), ("iso_f64", "hernquist"), ("per_f32", "zeldovich"),
         ("per_f64", "zeldovich")]


def _case(kind):
    if kind == "hernquist":
        p = ics.hernquist(n=3000, seed=5)
        return p.pos, p.vel, p.mass, 0.0, 0.02
    p = ics.zeldovich_box(n_side=20, seed=6)
    return p.pos, p.vel, p.mass, p.box, p.softening


def _restated(ref, fsize, pos, vel, mass):
    """The kicks and the drift of the harness's update sequence, restated."""
    ft = port.ftype(fsize)
    ids = ref["perm"]
    acc = vel.astype(ft)[:, ids]                   # Acc = Vel, in sorted order
    m = mass.astype(ft)[ids]
    order = np.flatnonzero(ids % 3 != 1)
    tree, top = ref["tree"], ref["topnodes"]
    for q in (4, 3):
        dt = (KICK_DT * (1 + ids % q) / q).astype(ft)
        dp = TU.particle_dp(m, dt, acc, fsize)
        tree, top = TU.kicks(tree, top, ref["tree_parent"], order, dp, fsize)
    upk = (tree, top)
    return upk, TU.drift(tree, top, DRIFT_DT, fsize)


ROOT = Path(__file__).resolve().parents[1]
_RUNS = {}


def _reference(variant, kind):
    """The harness's update run (cached: two tests read it)."""
    if not refrun.available(variant):
        pytest.skip(f"oracle/_ref/{variant} not built")
    if variant not in _RUNS:
        pos, vel, mass, box, soft = _case(kind)
        _RUNS[variant] = (refrun.run(variant, "update", pos, vel, mass, box=box, softening=soft,
                                     origin=(DRIFT_DT, 0.0, 0.0), size=KICK_DT),
                          pos, vel, mass, box, soft)
    return _RUNS[variant]


@pytest.mark.parametrize("variant,kind", CASES)
def test_tree_update_matches_reference(variant, kind):
    ref, pos, vel, mass, box, soft = _reference(variant, kind)
    fsize = ref["float_size"]
    (kt, ktop), (dt_, dtop) = _restated(ref, fsize, pos, vel, mass)
    # the kicks reached nodes and top nodes, and the drift moved them
    assert ((ref["upk_tree"]["Bitfield"] & TU.UPDATED) != 0).sum() > len(ref["tree"]) // 4
    assert (ref["upk_top"]["Level"] < 0).any()
    assert not np.array_equal(ref["upd_tree"]["CoM"], ref["tree"]["CoM"])
    assert_struct_equal(kt, ref["upk_tree"], TREE_FIELDS, "tree after the kicks")
    assert_struct_equal(ktop, ref["upk_top"], TOP_FIELDS, "top nodes after the kicks")
    assert_struct_equal(dt_, ref["upd_tree"], TREE_FIELDS, "tree after the drift")
    assert_struct_equal(dtop, ref["upd_top"], TOP_FIELDS, "top nodes after the drift")

    # the walks on the updated tree
    ft = port.ftype(fsize)
    pos_s, mass_s = pos.astype(ft)[:, ref["perm"]], mass.astype(ft)[ref["perm"]]
    prm = port.WalkParams(gravity=float(ref["gravity"][0]), softening=soft,
                          domain_size=float(ref["domain_size"][0]), boxsize=box, open_bh=0.25,
                          open_rel=0.005, use_bh=1, vector_size=64)
    ew = oracle_ewald_tables(fsize, box) if box > 0 else None
    last = np.zeros(len(mass_s), ft)
    for name, use_bh in (("bh", 1), ("rel", 0)):
        prm.use_bh = use_bh
        g, cg = port.walk("gravity", pos_s, mass_s, last, dtop, dt_, prm, fsize=fsize)
        gacc = g.astype(ft)
        if ew is not None:
            e, _ = port.walk("ewald", pos_s, mass_s, last, dtop, dt_, prm, ew, fsize=fsize)
            gacc = (gacc.astype(np.float64) + e).astype(ft)
        got, want = gacc.astype(np.float64), ref[name + "_gacc"]
        assert np.array_equal(got, want), f"{name}: max diff {np.abs(got - want).max()}"
        if name == "bh":
            last = np.sqrt(gacc[0] * gacc[0] + gacc[1] * gacc[1] + gacc[2] * gacc[2]).astype(ft)


@pytest.fixture(scope="module")
def host_lib(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("nvcc not found")
    out = tmp_path_factory.mktemp("tree_update_host") / "libtuhost.so"
    subprocess.run([nvcc, "-x", "cu", "-std=c++17", "-O2", "-shared", "-Xcompiler",
                    "-fPIC,-ffp-contract=off", "-I", str(ROOT / "include"),
                    str(ROOT / "tests" / "tree_update_host.cu"), "-o", str(out)],
                   check=True, capture_output=True)
    return C.CDLL(str(out))


@pytest.mark.parametrize("variant,kind", CASES)
def test_library_node_functions_match_reference(host_lib, variant, kind):
    """The per-node functions the kernels run (first particle of a node,
    active slots by the scan of the active flags, dp, node and top-node
    kicks and drifts), looped on the CPU, against the reference."""
    ref, pos, vel, mass, box, soft = _reference(variant, kind)
    fsize = ref["float_size"]
    ft = port.ftype(fsize)
    ids = ref["perm"]
    n = len(ids)
    flag = (ids % 3 != 1).astype(np.int32)
    off = np.zeros(n, np.int32)
    off[1:] = np.cumsum(flag)[:-1]
    na = int(flag.sum())
    m = np.ascontiguousarray(mass.astype(ft)[ids])
    acc = np.ascontiguousarray(vel.astype(ft)[:, ids])
    tree, top = ref["tree"].copy(), ref["topnodes"].copy()
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    for q in (4, 3):
        dt = np.ascontiguousarray((KICK_DT * (1 + ids % q) / q).astype(ft))
        dp = np.zeros((3, n), ft)
        host_lib.tu_host_dp(C.c_int(fsize), C.c_int64(n), p(flag), p(off), p(m), p(dt), p(acc),
                            p(dp), C.c_int64(n))
        bad = host_lib.tu_host_kick(C.c_int(fsize), p(tree), C.c_int64(len(tree)), p(top),
                                    C.c_int(len(top)), p(off), C.c_int64(n), C.c_int64(na), p(dp),
                                    C.c_int64(n))
        assert bad == 0
    assert_struct_equal(tree, ref["upk_tree"], TREE_FIELDS, "tree after the kicks")
    assert_struct_equal(top, ref["upk_top"], TOP_FIELDS, "top nodes after the kicks")
    host_lib.tu_host_drift(C.c_int(fsize), p(tree), C.c_int64(len(tree)), p(top), C.c_int(len(top)),
                           C.c_double(DRIFT_DT))
    assert_struct_equal(tree, ref["upd_tree"], TREE_FIELDS, "tree after the drift")
    assert_struct_equal(top, ref["upd_top"], TOP_FIELDS, "top nodes after the drift")


def test_kicks_reach_top_node_without_subtree():
    """A particle of a top node without subtree (Tree_Parent = -t - 1) kicks
    only that top node (tree_update.c:42-43)."""
    tree = np.zeros(1, refrun.TREE_DTYPE[4])
    top = np.zeros(2, refrun.TOPNODE_DTYPE)
    top["Level"] = 2
    top["Mass"] = 2.0
    dp = np.array([[1.0], [2.0], [4.0]], np.float32)
    _, t = TU.kicks(tree, top, np.array([-2], np.int32), [0], dp, 4)
    assert list(t["Level"]) == [2, -2]
    np.testing.assert_array_equal(t["Dp"][1], [0.5, 1.0, 2.0])
    _, t2 = TU.drift(tree, t, 2.0, 4)
    assert list(t2["Level"]) == [2, 2]
    np.testing.assert_array_equal(t2["CoM"][1], [1.0, 2.0, 4.0])
    np.testing.assert_array_equal(t2["Dp"][1], [0, 0, 0])
