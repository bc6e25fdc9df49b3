"""The oracle restatement against the golden fixtures produced by the real
reference (tests/golden/make_golden.py). Everything here is exact: keys,
sort permutation, top nodes, every tree field, Tree_Parent and the
accelerations and interaction counts of both walks."""
import numpy as np
import pytest

import port
from pipeline import oracle_pipeline, oracle_ewald_tables, assert_struct_equal
from tree_audit import audit

FORCE_CASES = ["hernquist_iso_f64", "hernquist_iso_f32", "box_per_f32", "zeldovich_per_f64",
               "box_per_f32_v32", "hernquist_iso_f64_v16"]
TREE_FIELDS = ["DNext", "Bitfield", "DUp", "Npart", "Pos", "Mass", "CoM", "Dp"]
TOP_FIELDS = ["Key", "Target", "Level", "First_Part", "Npart", "Pos", "Mass", "CoM"]


@pytest.mark.parametrize("fsize,variant", [(4, "iso_f32"), (8, "iso_f64")])
def test_keys_grid(golden_dir, fsize, variant):
    g = np.load(golden_dir / "keys_grid.npz")
    std, rev = port.peano_keys(g["pos"], (0.0, 0.0, 0.0), 1.0, fsize)
    assert np.array_equal(std, g[f"{variant}_std"])
    assert np.array_equal(rev, g[f"{variant}_rev"])


def test_keys_levels_consistent(golden_dir):
    """The standard and reversed keys carry the same triplets (peano.c)."""
    g = np.load(golden_dir / "keys_grid.npz")
    std, rev = g["iso_f64_std"], g["iso_f64_rev"]
    for i in range(0, len(std), 7):
        s = (int(std[i, 0]) << 64) | int(std[i, 1])
        r = (int(rev[i, 0]) << 64) | int(rev[i, 1])
        for lvl in range(1, 42):
            assert (s >> (128 - 3 * lvl)) & 7 == (r >> (3 * lvl)) & 7


@pytest.fixture(scope="module")
def ewald_cache():
    return {}


@pytest.mark.parametrize("case", FORCE_CASES)
def test_pipeline_matches_reference(golden_dir, case, ewald_cache):
    g = np.load(golden_dir / f"{case}.npz")
    fsize = int(g["float_size"])
    box = float(g["box"])
    ew = None
    if box > 0:
        key = (fsize, box)
        if key not in ewald_cache:
            ewald_cache[key] = oracle_ewald_tables(fsize, box)
        ew = ewald_cache[key]
    vsize = int(g["vector_size"]) if "vector_size" in g.files else 64
    o = oracle_pipeline(g["pos_in"], g["mass_in"], g["domain_origin"], float(g["domain_size"][0]),
                        fsize, box=box, softening=float(g["softening"]),
                        gravity=float(g["gravity"][0]), ewald=ew, vector_size=vsize)
    assert np.array_equal(o["perm"], g["perm"])
    assert np.array_equal(o["std_key"], g["std_key"])
    assert np.array_equal(o["rev_key"], g["rev_key"])
    assert_struct_equal(o["top"], g["topnodes"], TOP_FIELDS, "topnodes")
    assert_struct_equal(o["tree"], g["tree"], TREE_FIELDS, "tree")
    assert np.array_equal(o["tree_parent"], g["tree_parent"])
    for name in ("bh", "rel"):
        assert np.array_equal(o[name + "_cost"], g[name + "_cost"].astype(o[name + "_cost"].dtype))
        ref = g[name + "_gacc"]
        got = o[name + "_gacc"].astype(np.float64)
        assert np.array_equal(got, ref), f"{name}: max diff {np.abs(got - ref).max()}"
        if box > 0:
            assert np.array_equal(o[name + "ew_gacc"].astype(np.float64), g[name + "ew_gacc"])
    assert np.array_equal(o["last_acc_mag"].astype(np.float64), g["last_acc_mag"])


def test_ewald_table_matches_reference_formula():
    """Table points against the direct evaluation of the same sums, and the
    folded symmetry the lookup relies on (odd in its own axis)."""
    fx, fy, fz, fp = port.ewald_table(n_ewald=8, potential=True)
    m = 9
    pts, ref = [], []
    for (i, j, k) in [(1, 2, 3), (8, 8, 8), (0, 5, 2), (7, 0, 0)]:
        pts.append((0.5 * i / 8, 0.5 * j / 8, 0.5 * k / 8))
        idx = (i * m + j) * m + k
        ref.append((fx[idx], fy[idx], fz[idx]))
    f = port.ewald_force(np.array(pts), nreal=4, nk=4)
    assert np.allclose(f, np.array(ref), rtol=0, atol=1e-15)
    fneg = port.ewald_force(-np.array(pts), nreal=4, nk=4)
    assert np.allclose(fneg, -f, atol=1e-12)


@pytest.mark.parametrize("case", ["hernquist_iso_f64", "hernquist_iso_f32", "zeldovich_per_f64"])
def test_potential_build_changes_nothing_else(golden_dir, case):
    """The reference built with GRAVITY_POTENTIAL (the *_pot fixtures) gives
    the same keys, order, tree and forces as without it, plus Grav_Pot."""
    a = np.load(golden_dir / f"{case}.npz")
    b = np.load(golden_dir / f"{case}_pot.npz")
    shared = [k for k in a.files if k in b.files]
    assert {"perm", "tree", "bh_gacc", "rel_gacc"} <= set(shared)
    for k in shared:
        assert np.array_equal(a[k], b[k]), k
    assert np.all(np.isfinite(b["bh_pot"])) and np.all(np.isfinite(b["rel_pot"]))


@pytest.mark.parametrize("case", ["hernquist_iso_f64_pot", "hernquist_iso_f32_pot",
                                  "zeldovich_per_f64_pot"])
def test_oracle_potential_matches_reference(golden_dir, case):
    """The restatement's potential (port.walk(potential=True)) against the
    reference built with GRAVITY_POTENTIAL, both passes, bit for bit: the
    gravity pass assigns Grav_Pot (tree_accel.c:122-124), the Ewald pass adds
    to it (tree_periodic.c:103-105)."""
    g = np.load(golden_dir / f"{case}.npz")
    fsize = int(g["float_size"])
    ft = port.ftype(fsize)
    box = float(g["box"])
    pos = g["pos_in"].astype(ft)[:, g["perm"]]
    mass = g["mass_in"].astype(ft)[g["perm"]]
    prm = port.WalkParams(gravity=float(g["gravity"][0]), softening=float(g["softening"]),
                          domain_size=float(g["domain_size"][0]), boxsize=box, open_bh=0.25,
                          open_rel=0.005, use_bh=1, vector_size=64)
    tabs = None
    if box > 0:
        fx, fy, fz, fp = port.ewald_table(potential=True)
        tabs = [(t.astype(ft).astype(np.float64) / (box * box)).astype(ft) for t in (fx, fy, fz)]
        tabs.append((fp.astype(ft).astype(np.float64) / box).astype(ft))
    for name, use_bh, last in (("bh", 1, np.zeros(len(mass), ft)),
                               ("rel", 0, g["last_acc_mag"].astype(ft))):
        prm.use_bh = use_bh
        _, _, pg = port.walk("gravity", pos, mass, last, g["topnodes"], g["tree"], prm,
                             fsize=fsize, potential=True)
        pot = pg.astype(ft)
        if box > 0:
            _, _, pe = port.walk("ewald", pos, mass, last, g["topnodes"], g["tree"], prm, tabs,
                                 fsize=fsize, potential=True)
            pot = (pot.astype(np.float64) + pe).astype(ft)
        ref = g[name + "_pot"]
        assert np.array_equal(pot.astype(np.float64), ref), \
            f"{name}: max diff {np.abs(pot.astype(np.float64) - ref).max()}"


@pytest.mark.parametrize("case", FORCE_CASES)
def test_tree_audit_on_reference_trees(golden_dir, case):
    """The reference's node audit (tree_build.c:620-685, tests/tree_audit.py)
    passes on the reference's own trees, and catches a mistake planted in a
    copy of one (Npart, DNext, CoM or a node centre changed)."""
    g = np.load(golden_dir / f"{case}.npz")
    fsize = int(g["float_size"])
    ft = port.ftype(fsize)
    pos = g["pos_in"].astype(ft)[:, g["perm"]]
    mass = g["mass_in"].astype(ft)[g["perm"]]
    size = float(g["domain_size"][0])
    vsize = int(g["vector_size"]) if "vector_size" in g.files else 64
    audit(g["tree"], g["topnodes"], pos, mass, size, fsize, vector_size=vsize)
    i = np.flatnonzero(g["tree"]["DNext"] > 0)[3]
    for field, k, delta in (("Npart", None, 1), ("DNext", None, 1), ("CoM", 0, 0.05 * size),
                            ("Pos", 1, 1e-4 * size)):
        bad = g["tree"].copy()
        if k is None:
            bad[field][i] += delta
        else:
            bad[field][i + 1, k] += delta
        with pytest.raises(AssertionError):
            audit(bad, g["topnodes"], pos, mass, size, fsize, vector_size=vsize)


@pytest.mark.parametrize("case", ["hernquist_iso_f32", "hernquist_iso_f64"])
def test_domain_matches_reference(golden_dir, case):
    """set_computational_domain restated (port.find_domain) against the
    reference's Domain.Origin/Size. The reference computes it twice before
    its first tree: in Setup_Domain_Decomposition on the input order, then,
    after that sort, in Domain_Decomposition on the PH order
    (domain.c:67-71, 150-172). Its Median leaves out the first particle of
    the current order (select.c:19-107), so the second pass differs from the
    first; the restatement reproduces the second bit for bit."""
    g = np.load(golden_dir / f"{case}.npz")
    fs = int(g["float_size"])
    pos = g["pos_in"].astype(port.ftype(fs))
    o1, s1 = port.find_domain(pos, fs)
    std, _ = port.peano_keys(pos, o1, s1, fs)
    perm = port.sort_keys(std)
    o2, s2 = port.find_domain(pos[:, perm], fs)
    assert np.array_equal(o2, g["domain_origin"]) and s2 == float(g["domain_size"][0])
    assert not np.array_equal(o1, o2)
