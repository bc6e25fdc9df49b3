"""CUDA path against the oracle and the reference's golden fixtures, through
the C ABI. Keys, sort permutation, top nodes, every tree field and
Tree_Parent must be bit-exact; so must the plain-form accelerations and
interaction counts (the plain form replays the reference's arithmetic) where
the Ewald table is the reference's own (FP32); the FP64 periodic walk is
compared within 1e-12 relative, because the GPU's erfc/exp/sin differ from
glibc's in the last bit of the FP64 table."""
import numpy as np
import pytest

import port
from pipeline import oracle_pipeline, oracle_ewald_tables, assert_struct_equal
from tandav_b200 import gravity as G
from tree_audit import audit
from tandav_b200 import ics

pytestmark = pytest.mark.gpu

TREE_FIELDS = ["DNext", "Bitfield", "DUp", "Npart", "Pos", "Mass", "CoM", "Dp"]
TOP_FIELDS = ["Key", "Target", "Level", "First_Part", "Npart", "Pos", "Mass", "CoM"]
FORCE_CASES = ["hernquist_iso_f64", "hernquist_iso_f32", "box_per_f32", "zeldovich_per_f64",
               "box_per_f32_v32", "hernquist_iso_f64_v16"]


def make_ctx(n, fsize, box=0.0, softening=0.01, gravity=43007.1, **kw):
    return G.GravityContext(max(n, 1024), float_bytes=fsize, periodic=box > 0, boxsize=box,
                            gravity=gravity, softening=softening, **kw)


@pytest.mark.parametrize("fsize,variant", [(4, "iso_f32"), (8, "iso_f64")])
def test_keys_grid(golden_dir, fsize, variant):
    g = np.load(golden_dir / "keys_grid.npz")
    pos = g["pos"]
    n = pos.shape[1]
    with make_ctx(n, fsize) as ctx:
        ctx.upload(pos, np.ones(n))
        ctx.set_domain((0.0, 0.0, 0.0), 1.0)
        ctx.peano_keys()
        assert np.array_equal(ctx.download(G.F_KEY)["key"], g[f"{variant}_std"])
        ctx.reverse_keys()
        assert np.array_equal(ctx.download(G.F_KEY)["key"], g[f"{variant}_rev"])


def gpu_pipeline(ctx, pos, mass, origin, size, exact=True):
    ctx.upload(pos, mass)
    ctx.set_domain(origin, size)
    ctx.peano_keys()
    perm = ctx.sort_particles()
    keys = ctx.download(G.F_KEY)["key"]
    ctx.top_nodes()
    ctx.tree_build(exact_moments=exact)
    tree, top = ctx.download_tree()
    return perm, keys, tree, top


_RAW_TABLE = {}


def reference_table(fsize):
    """The reference's raw Float tables (the oracle's FP64 sums, verified
    bit-identical to the reference's ./ewald_tables.dat), as a drop-in host
    would read them from that file."""
    if fsize not in _RAW_TABLE:
        fx, fy, fz, fp = port.ewald_table(potential=True)
        _RAW_TABLE[fsize] = [t.astype(port.ftype(fsize)) for t in (fx, fy, fz, fp)]
    return _RAW_TABLE[fsize]


def walks(ctx, periodic, fsize):
    parts = G.WALK_GRAVITY | (G.WALK_EWALD if periodic else 0)
    if periodic:
        ctx.upload_ewald_table(*reference_table(fsize))
    ctx.zero_accel()
    ctx.walk(G.FORM_PLAIN, use_bh=True, parts=parts)
    bh = ctx.download(G.F_GRAV_ACC | G.F_COST)
    ctx.save_last_accel()
    last = ctx.download(G.F_LAST_ACC)["last_acc_mag"]
    ctx.walk(G.FORM_PLAIN, use_bh=False, parts=parts)
    rel = ctx.download(G.F_GRAV_ACC | G.F_COST)
    return bh, last, rel


@pytest.mark.parametrize("case", FORCE_CASES)
def test_pipeline_matches_reference_golden(golden_dir, case):
    g = np.load(golden_dir / f"{case}.npz")
    fsize = int(g["float_size"])
    box = float(g["box"])
    n = len(g["mass_in"])
    vsize = int(g["vector_size"]) if "vector_size" in g.files else 64
    with make_ctx(n, fsize, box=box, softening=float(g["softening"]),
                  gravity=float(g["gravity"][0]), vector_size=vsize) as ctx:
        perm, keys, tree, top = gpu_pipeline(ctx, g["pos_in"], g["mass_in"], g["domain_origin"],
                                             float(g["domain_size"][0]))
        assert np.array_equal(perm, g["perm"])
        assert np.array_equal(keys, g["std_key"])
        assert_struct_equal(top, g["topnodes"], TOP_FIELDS, "topnodes")
        assert_struct_equal(tree, g["tree"], TREE_FIELDS, "tree")
        assert np.array_equal(ctx.download(G.F_TREE_PARENT)["tree_parent"], g["tree_parent"])
        bh, last, rel = walks(ctx, box > 0, fsize)
        for name, got in (("bh", bh), ("rel", rel)):
            assert np.array_equal(got["cost"].astype(np.float64), g[name + "_cost"]), name
            ref = g[name + "_gacc"]
            a = got["grav_acc"].astype(np.float64)
            assert np.array_equal(a, ref), f"{name}: max diff {np.abs(a - ref).max()}"
        assert np.array_equal(last.astype(np.float64), g["last_acc_mag"])
        ctx.reverse_keys()
        assert np.array_equal(ctx.download(G.F_KEY)["key"], g["rev_key"])


def test_config1_hernquist_65536_fp64_vs_reference():
    """The CPU-runnable configuration exactly: an isolated Hernquist halo of
    65,536 equal-mass particles (a = 1, truncated at 100 a, eps = 0.01 a), FP64,
    one tree build and both passes -- Barnes-Hut (theta^2 0.25), then the
    relative criterion (errtol 0.005) with |a_old| from the first pass
    (accel.c:15-71). The reference itself (oracle/_ref/iso_f64, the unmodified
    sources) runs on the same input here; keys, permutation, top nodes, every
    tree field, Tree_Parent, both passes' accelerations and interaction counts
    and Last_Acc_Mag must equal its output bit for bit."""
    import refrun
    if not refrun.available("iso_f64"):
        pytest.skip("reference harness oracle/_ref/iso_f64 not built (make -C oracle ref)")
    p = ics.hernquist(n=65536, seed=31)
    r = refrun.run("iso_f64", "force", p.pos, p.vel, p.mass, softening=p.softening, flags=3)
    assert r["float_size"] == 8
    with make_ctx(p.n, 8, softening=p.softening, gravity=float(r["gravity"][0])) as ctx:
        perm, keys, tree, top = gpu_pipeline(ctx, p.pos, p.mass, r["domain_origin"],
                                             float(r["domain_size"][0]))
        assert np.array_equal(perm, r["perm"])
        assert np.array_equal(keys, r["std_key"])
        assert_struct_equal(top, r["topnodes"], TOP_FIELDS, "topnodes")
        assert_struct_equal(tree, r["tree"], TREE_FIELDS, "tree")
        assert np.array_equal(ctx.download(G.F_TREE_PARENT)["tree_parent"], r["tree_parent"])
        bh, last, rel = walks(ctx, False, 8)
        for name, got in (("bh", bh), ("rel", rel)):
            assert np.array_equal(got["cost"].astype(np.float64), r[name + "_cost"]), name
            a = got["grav_acc"].astype(np.float64)
            assert np.array_equal(a, r[name + "_gacc"]), \
                f"{name}: max diff {np.abs(a - r[name + '_gacc']).max()}"
        assert np.array_equal(last.astype(np.float64), r["last_acc_mag"])
        ctx.reverse_keys()
        assert np.array_equal(ctx.download(G.F_KEY)["key"], r["rev_key"])


BALANCED_CASES = ["decomp_hernquist_iso_f64_t3", "decomp_clumpy_per_f32_t8"]


@pytest.mark.parametrize("case", BALANCED_CASES)
def test_balanced_decomposition_matches_reference(golden_dir, case):
    """Top nodes balanced over NTask = 3 and 8 targets by the P.Cost of a
    first force computation, as the reference's second Domain_Decomposition
    makes them (domain.c:67-145, 151-156; levels 2 to 6, up to several hundred
    top nodes), then the tree and both passes on them: permutation, keys, top
    nodes, every tree field, Tree_Parent, forces and interaction counts equal
    the reference's bit for bit."""
    g = np.load(golden_dir / f"{case}.npz")
    fsize, box = int(g["float_size"]), float(g["box"])
    n = len(g["mass_in"])
    cost = np.empty(n)
    cost[g["id_in"].astype(np.int64)] = g["cost_in"]
    with make_ctx(n, fsize, box=box, softening=float(g["softening"]),
                  gravity=float(g["gravity"][0])) as ctx:
        ctx.set_domain_decomposition(int(g["ntask"]))
        ctx.upload(g["pos_in"], g["mass_in"], cost=cost)
        ctx.set_domain(g["domain_origin"], float(g["domain_size"][0]))
        ctx.peano_keys()
        perm = ctx.sort_particles()
        keys = ctx.download(G.F_KEY)["key"]
        ntop = ctx.top_nodes()
        assert ctx.decomposition_rounds() > 0
        ctx.tree_build(exact_moments=True)
        tree, top = ctx.download_tree()
        assert ntop == len(g["topnodes"])
        assert np.array_equal(perm, g["perm"])
        assert np.array_equal(keys, g["std_key"])
        assert_struct_equal(top, g["topnodes"], TOP_FIELDS, "topnodes")
        assert_struct_equal(tree, g["tree"], TREE_FIELDS, "tree")
        assert np.array_equal(ctx.download(G.F_TREE_PARENT)["tree_parent"], g["tree_parent"])
        bh, last, rel = walks(ctx, box > 0, fsize)
        for name, got in (("bh", bh), ("rel", rel)):
            assert np.array_equal(got["cost"].astype(np.float64), g[name + "_cost"]), name
            a = got["grav_acc"].astype(np.float64)
            assert np.array_equal(a, g[name + "_gacc"]), \
                f"{name}: max diff {np.abs(a - g[name + '_gacc']).max()}"
        assert np.array_equal(last.astype(np.float64), g["last_acc_mag"])


def test_balanced_decomposition_vs_oracle_at_size():
    """2^19 particles in clumps (FP32, periodic) balanced over 8 targets with
    synthetic costs: ~5e4 interactions per particle in a slab of 12 % of the
    box, 1-100 elsewhere, so the slab's cells are split down to level 7 (1177
    top nodes). The bunch costs reach 10^9, far above 2^24, so the float
    partial sums of the thread shares round, in the same order on both
    sides. Top nodes, tree and Tree_Parent equal the oracle's
    (oracle/decomposition.py and the restated build)."""
    p = ics.random_box(1 << 19, box=1000.0, seed=45, clumps=11)
    h = np.arange(p.n, dtype=np.uint64) * 2654435761
    cost = np.where(p.pos[0] < 120.0, 50000 - (h % 1000), h % 100 + 1).astype(np.float64)
    ew = oracle_ewald_tables(4, p.box)
    o = oracle_pipeline(p.pos, p.mass, np.zeros(3), p.box, 4, box=p.box, softening=p.softening,
                        passes=("bh",), ntask=8, cost=cost, ewald=ew)
    assert len(o["top"]) > 1000
    parts = G.WALK_GRAVITY | G.WALK_EWALD
    with make_ctx(p.n, 4, box=p.box, softening=p.softening) as ctx:
        ctx.set_domain_decomposition(8)
        ctx.upload(p.pos, p.mass, cost=cost)
        ctx.set_domain((0.0, 0.0, 0.0), p.box)
        ctx.peano_keys()
        perm = ctx.sort_particles()
        ctx.top_nodes()
        ctx.tree_build(exact_moments=True)
        tree, top = ctx.download_tree()
        assert np.array_equal(perm, o["perm"])
        assert_struct_equal(top, o["top"], TOP_FIELDS, "topnodes")
        assert_struct_equal(tree, o["tree"], TREE_FIELDS, "tree")
        assert np.array_equal(ctx.download(G.F_TREE_PARENT)["tree_parent"], o["tree_parent"])
        # the plain walk over 1177 top nodes (read through L1, not staged)
        ctx.upload_ewald_table(*reference_table(4))
        ctx.zero_accel()
        ctx.walk(G.FORM_PLAIN, use_bh=True, parts=parts)
        got = ctx.download(G.F_GRAV_ACC | G.F_COST)
        assert np.array_equal(got["cost"], o["bh_cost"])
        assert np.array_equal(got["grav_acc"].astype(np.float64), o["bh_gacc"].astype(np.float64))
        # the group walks push their roots in chunks of 256
        ctx.ewald_init()
        ctx.zero_accel()
        ctx.walk(G.FORM_GROUP, use_bh=True, parts=parts)
        ga = ctx.download(G.F_GRAV_ACC)["grav_acc"].astype(np.float64)
        assert np.all(np.isfinite(ga)) and np.all(np.abs(ga).sum(0) > 0)


RANDOM_CASES = [
    ("hernquist", 8, 32768),
    ("hernquist", 4, 65536),
    ("clumpy_box", 4, 40000),
    ("zeldovich", 4, 32 ** 3),
]


def make_case(kind, n):
    if kind == "hernquist":
        p = ics.hernquist(n=n, seed=21)
        c = np.median(p.pos, axis=1)
        size = 2.001 * np.abs(p.pos - c[:, None]).max()
        return p, c - 0.5 * size, size
    if kind == "clumpy_box":
        p = ics.random_box(n, box=2000.0, seed=22, clumps=9)
    else:
        p = ics.zeldovich_box(n_side=round(n ** (1 / 3)), seed=23)
    return p, np.zeros(3), p.box


@pytest.mark.parametrize("kind,fsize,n", RANDOM_CASES)
def test_tree_and_plain_walk_vs_oracle(kind, fsize, n):
    p, origin, size = make_case(kind, n)
    ew = oracle_ewald_tables(fsize, p.box) if p.box > 0 else None
    o = oracle_pipeline(p.pos, p.mass, origin, size, fsize, box=p.box, softening=p.softening,
                        ewald=ew, passes=("bh", "rel"))
    with make_ctx(p.n, fsize, box=p.box, softening=p.softening) as ctx:
        perm, keys, tree, top = gpu_pipeline(ctx, p.pos, p.mass, origin, size)
        assert np.array_equal(perm, o["perm"])
        assert_struct_equal(top, o["top"], TOP_FIELDS, "topnodes")
        assert_struct_equal(tree, o["tree"], TREE_FIELDS, "tree")
        assert np.array_equal(ctx.download(G.F_TREE_PARENT)["tree_parent"], o["tree_parent"])
        # both passes: Barnes-Hut, then the relative criterion with |a_old|
        # from the first (accel.c:15-71)
        bh, last, rel = walks(ctx, p.box > 0, fsize)
        for name, got in (("bh", bh), ("rel", rel)):
            assert np.array_equal(got["cost"], o[name + "_cost"]), name
            a, ref = got["grav_acc"].astype(np.float64), o[name + "_gacc"].astype(np.float64)
            assert np.array_equal(a, ref), f"{name}: max diff {np.abs(a - ref).max()}"
        assert np.array_equal(last, o["last_acc_mag"])


def test_fast_moments_close_to_exact():
    p, origin, size = make_case("zeldovich", 32 ** 3)
    with make_ctx(p.n, 4, box=p.box, softening=p.softening) as ctx:
        _, _, exact, top_e = gpu_pipeline(ctx, p.pos, p.mass, origin, size, exact=True)
        _, _, fast, top_f = gpu_pipeline(ctx, p.pos, p.mass, origin, size, exact=False)
    assert_struct_equal(exact, fast, ["DNext", "Bitfield", "DUp", "Npart", "Pos"], "topology")
    assert np.allclose(exact["Mass"], fast["Mass"], rtol=1e-5)
    assert np.allclose(exact["CoM"], fast["CoM"], rtol=0, atol=1e-4 * p.box)


@pytest.mark.parametrize("case", ["hernquist_iso_f32", "hernquist_iso_f64", "hernquist_2^18"])
def test_find_domain_matches_reference(golden_dir, case):
    """tvg_find_domain as the reference's setup runs it: on the input order,
    then (after the keys and the sort) on the PH order. The golden cases
    match the reference's Domain.Origin/Size bit for bit; a 2^18 sphere
    matches the restatement (port.find_domain) in FP32."""
    if case.startswith("hernquist_iso"):
        g = np.load(golden_dir / f"{case}.npz")
        fs, pos, mass = int(g["float_size"]), g["pos_in"], g["mass_in"]
        want_o, want_s = g["domain_origin"], float(g["domain_size"][0])
    else:
        p = ics.hernquist(n=1 << 18, seed=9)
        fs, pos, mass = 4, p.pos, p.mass
        pf = pos.astype(np.float32)
        o1, s1 = port.find_domain(pf, 4)
        std, _ = port.peano_keys(pf, o1, s1, 4)
        want_o, want_s = port.find_domain(pf[:, port.sort_keys(std)], 4)
    with make_ctx(pos.shape[1], fs) as ctx:
        ctx.upload(pos, mass)
        ctx.find_domain()                         # Setup_Domain_Decomposition
        ctx.peano_keys()
        ctx.sort_particles()
        o, s = ctx.find_domain()                  # Domain_Decomposition
    assert np.array_equal(o, want_o) and s == want_s


@pytest.mark.parametrize("case", ["hernquist_iso_f32", "hernquist_iso_f64"])
def test_isolated_setup_finds_the_reference_domain(golden_dir, case):
    """The isolated pipeline from the input order with TVG_CFG_FIND_DOMAIN, run
    as the reference's setup runs it: tvg_find_domain, keys and sort
    (Setup_Domain_Decomposition), then a force step that finds the domain
    again on the PH order (Domain_Decomposition), builds and walks. The
    particle order, the top nodes, every tree field and the Barnes-Hut
    accelerations equal the reference's golden output bit for bit, with no
    domain given by the host."""
    g = np.load(golden_dir / f"{case}.npz")
    fsize = int(g["float_size"])
    n = len(g["mass_in"])
    with make_ctx(n, fsize, softening=float(g["softening"]), gravity=float(g["gravity"][0]),
                  flags=G.CFG_FIND_DOMAIN) as ctx:
        ctx.upload(g["pos_in"], g["mass_in"], ids=np.arange(n, dtype=np.uint32))
        ctx.find_domain()
        ctx.peano_keys()
        ctx.sort_particles()
        ctx.force_step(form=G.FORM_PLAIN, use_bh=True, parts=G.WALK_GRAVITY)
        d = ctx.download(G.F_ID | G.F_GRAV_ACC)
        tree, top = ctx.download_tree()
    assert np.array_equal(d["id"], g["perm"])
    assert_struct_equal(top, g["topnodes"], TOP_FIELDS, "topnodes")
    assert_struct_equal(tree, g["tree"], TREE_FIELDS, "tree")
    assert np.array_equal(d["grav_acc"].astype(np.float64), g["bh_gacc"])


def test_keys_sort_and_tree_of_the_256_box():
    """The 256^3 benchmark box (16.7M particles): every 128-bit key, the sort
    permutation, the top nodes, every field of the 913k tree nodes and
    Tree_Parent bit for bit against the oracle (C restatement, pinned to the
    reference on the golden cases)."""
    p, origin, size = make_case("zeldovich", 256 ** 3)
    pos_f = p.pos.astype(np.float32)
    std, rev = port.peano_keys(pos_f, origin, size, 4)
    perm_o = port.sort_keys(std)
    pos_s, mass_s = pos_f[:, perm_o], p.mass.astype(np.float32)[perm_o]
    top_o = port.top_nodes(std[perm_o], pos_s, origin, size, 4)
    tree_o, top_o, parent_o = port.tree_build(rev[perm_o], pos_s, mass_s, size, top_o, 4)
    with make_ctx(p.n, 4, box=p.box, softening=p.softening) as ctx:
        perm, keys, tree, top = gpu_pipeline(ctx, p.pos, p.mass, origin, size, exact=True)
        parent = ctx.download(G.F_TREE_PARENT)["tree_parent"]
    assert np.array_equal(perm, perm_o)
    assert np.array_equal(keys, std[perm_o])
    assert_struct_equal(top, top_o, TOP_FIELDS, "topnodes")
    assert_struct_equal(tree, tree_o, TREE_FIELDS, "tree")
    assert np.array_equal(parent, parent_o)


@pytest.mark.parametrize("kind,fsize,n,vsize", [("zeldovich", 4, 64 ** 3, 32),
                                               ("zeldovich", 4, 64 ** 3, 8),
                                               ("hernquist", 8, 1 << 17, 32),
                                               ("clumpy_box", 4, 1 << 17, 16)])
def test_tree_vs_oracle_at_other_vector_sizes(kind, fsize, n, vsize):
    """VECTOR_SIZE (bundle size) is a compile-time constant of the reference
    (64 by default); the build takes it from the context's configuration.
    Top nodes, every tree field and Tree_Parent at smaller bundle sizes equal
    the oracle's build with the same VECTOR_SIZE, and the tree passes the
    node audit."""
    p, origin, size = make_case(kind, n)
    ft = port.ftype(fsize)
    pos_f = p.pos.astype(ft)
    std, rev = port.peano_keys(pos_f, origin, size, fsize)
    perm_o = port.sort_keys(std)
    pos_s, mass_s = pos_f[:, perm_o], p.mass.astype(ft)[perm_o]
    top_o = port.top_nodes(std[perm_o], pos_s, origin, size, fsize)
    tree_o, top_o, parent_o = port.tree_build(rev[perm_o], pos_s, mass_s, size, top_o, fsize,
                                              vector_size=vsize)
    with make_ctx(p.n, fsize, box=p.box, softening=p.softening, vector_size=vsize) as ctx:
        perm, keys, tree, top = gpu_pipeline(ctx, p.pos, p.mass, origin, size, exact=True)
        parent = ctx.download(G.F_TREE_PARENT)["tree_parent"]
    assert np.array_equal(perm, perm_o)
    assert_struct_equal(top, top_o, TOP_FIELDS, "topnodes")
    assert_struct_equal(tree, tree_o, TREE_FIELDS, "tree")
    assert np.array_equal(parent, parent_o)
    audit(tree, top, pos_s, mass_s, size, fsize, vector_size=vsize)


@pytest.mark.parametrize("kind,fsize,n,exact", [("zeldovich", 4, 128 ** 3, True),
                                               ("zeldovich", 4, 128 ** 3, False),
                                               ("hernquist", 8, 1 << 20, True),
                                               ("zeldovich", 4, 256 ** 3, True)])
def test_tree_audit_large(kind, fsize, n, exact):
    """The reference's node audit (tree_build.c:620-685, tests/tree_audit.py)
    over every node of trees built on the GPU at sizes beyond the oracle
    comparisons, up to the 256^3 benchmark box: branches against DNext,
    contiguous particle ranges and Npart, mass and centre of mass (exact
    Float sums or FP64 warp sums), octant geometry, every particle inside its
    bundle's cube (apart from the cubes the reference's own centre rule
    moves, which the audit finds exactly; 355 nodes in this 256^3 box)."""
    p, origin, size = make_case(kind, n)
    ft = port.ftype(fsize)
    with make_ctx(p.n, fsize, box=p.box, softening=p.softening) as ctx:
        perm, _, tree, top = gpu_pipeline(ctx, p.pos, p.mass, origin, size, exact=exact)
    figures = audit(tree, top, p.pos.astype(ft)[:, perm], p.mass.astype(ft)[perm], size, fsize)
    print(kind, n, "exact" if exact else "fast", figures)


@pytest.mark.parametrize("fsize", [4, 8])
def test_ewald_table_vs_oracle(fsize):
    box = 1000.0
    with make_ctx(1024, fsize, box=box) as ctx:
        ctx.upload(np.full((3, 4), 1.0), np.ones(4))
        ctx.ewald_init()
        fx, fy, fz, fp = ctx.download_ewald_table()
    ox, oy, oz, op = port.ewald_table(potential=True)
    ft = port.ftype(fsize)
    for name, got, ref in (("fx", fx, ox), ("fy", fy, oy), ("fz", fz, oz), ("fp", fp, op)):
        # the same FP64 sums with the GPU's erfc/exp/sin/cos: the terms cancel
        # to ~1e-3 of their size, so the last FP64 bits differ; stored in
        # Float they agree to within one Float ulp of the table's scale
        r = ref.astype(ft).astype(np.float64)
        scale = np.abs(ref).max()
        err = np.abs(got.astype(np.float64) - r)
        # FP64: the near-origin terms are ~1e4, so one FP64 ulp of those is ~1e-12
        tol = 1e-10 if fsize == 8 else float(np.spacing(np.float32(scale)))
        assert err.max() <= tol, f"{name}: max err {err.max()} > {tol}"


def test_sort_long_runs_of_equal_high_key_words():
    """Particles packed into cells of the 21st level share the high 64 bits of
    their Peano-Hilbert keys: the radix passes leave such runs (here of 20000,
    5000 and 300 particles) in input order, and the tie pass orders each by
    the low words. The permutation is the oracle's full 128-bit sort."""
    rng = np.random.default_rng(17)
    L = 1.0
    pos = [rng.uniform(0, L, (3, 150000))]
    for n_run in (20000, 5000, 300):
        cell = L / 2 ** 21
        corner = np.floor(rng.uniform(0.1, 0.9, 3) / cell) * cell
        pos.append(corner[:, None] + rng.uniform(0.1, 0.9, (3, n_run)) * cell)
    pos = np.concatenate(pos, axis=1)
    n = pos.shape[1]
    std, _ = port.peano_keys(pos, (0.0, 0.0, 0.0), L, 8)
    perm_o = port.sort_keys(std)
    assert len(np.unique(std[:, 0])) < n - 25000            # the runs are there
    with make_ctx(n, 8) as ctx:
        ctx.upload(pos, np.ones(n))
        ctx.set_domain((0.0, 0.0, 0.0), L)
        ctx.peano_keys()
        perm = ctx.sort_particles()
        keys = ctx.download(G.F_KEY)["key"]
    assert np.array_equal(perm, perm_o)
    assert np.array_equal(keys, std[perm_o])


def test_coincident_particles_reported():
    # enough particles that every top node gets a subtree (> 64 particles)
    p = ics.random_box(20000, box=100.0, seed=3)
    p.pos[:, 1] = p.pos[:, 0]
    with make_ctx(p.n, 4, box=p.box) as ctx:
        ctx.upload(p.pos, p.mass)
        ctx.set_domain((0.0, 0.0, 0.0), p.box)
        ctx.peano_keys()
        ctx.sort_particles()
        ctx.top_nodes()
        with pytest.raises(G.TvgError) as e:
            ctx.tree_build()
        assert e.value.code == 6


def test_nonfinite_position_reported():
    p = ics.random_box(1000, box=100.0, seed=4)
    p.pos[1, 17] = np.nan
    with make_ctx(p.n, 4, box=p.box) as ctx:
        ctx.upload(p.pos, p.mass)
        ctx.set_domain((0.0, 0.0, 0.0), p.box)
        with pytest.raises(G.TvgError) as e:
            ctx.peano_keys()
        assert e.value.code == 5


def test_state_errors():
    with make_ctx(1024, 4) as ctx:
        ctx.upload(np.random.default_rng(0).uniform(0, 1, (3, 100)), np.ones(100))
        with pytest.raises(G.TvgError) as e:
            ctx.peano_keys()                     # no domain
        assert e.value.code == 7
        ctx.set_domain((0.0, 0.0, 0.0), 1.0)
        with pytest.raises(G.TvgError) as e:
            ctx.walk()                           # no tree
        assert e.value.code == 7


POT_CASES = ["hernquist_iso_f64_pot", "hernquist_iso_f32_pot", "zeldovich_per_f64_pot"]


@pytest.mark.parametrize("case", POT_CASES)
def test_potential_matches_reference_golden(golden_dir, case):
    """TVG_CFG_POTENTIAL: Grav_Pot of the plain form (gravity + Ewald) bit for
    bit against the reference built with GRAVITY_POTENTIAL, both passes; the
    forces stay the reference's; the group form refuses the flag."""
    g = np.load(golden_dir / f"{case}.npz")
    fsize = int(g["float_size"])
    box = float(g["box"])
    n = len(g["mass_in"])
    with make_ctx(n, fsize, box=box, softening=float(g["softening"]), gravity=float(g["gravity"][0]),
                  flags=G.CFG_POTENTIAL) as ctx:
        perm, _, tree, _ = gpu_pipeline(ctx, g["pos_in"], g["mass_in"], g["domain_origin"],
                                        float(g["domain_size"][0]))
        assert np.array_equal(perm, g["perm"])
        assert_struct_equal(tree, g["tree"], TREE_FIELDS, "tree")
        parts = G.WALK_GRAVITY | (G.WALK_EWALD if box > 0 else 0)
        if box > 0:
            ctx.upload_ewald_table(*reference_table(fsize))
        ctx.zero_accel()
        ctx.walk(G.FORM_PLAIN, use_bh=True, parts=parts)
        bh = ctx.download(G.F_GRAV_ACC | G.F_GRAV_POT)
        ctx.save_last_accel()
        ctx.walk(G.FORM_PLAIN, use_bh=False, parts=parts)
        rel = ctx.download(G.F_GRAV_ACC | G.F_GRAV_POT)
        for name, got in (("bh", bh), ("rel", rel)):
            a = got["grav_acc"].astype(np.float64)
            assert np.array_equal(a, g[name + "_gacc"]), name
            p, ref = got["grav_pot"].astype(np.float64), g[name + "_pot"]
            assert np.array_equal(p, ref), f"{name}: max diff {np.abs(p - ref).max()}"
        with pytest.raises(G.TvgError):
            ctx.walk(G.FORM_GROUP, use_bh=False, parts=parts)


@pytest.mark.parametrize("kind,fsize,n", [("hernquist", 8, 32768), ("zeldovich", 4, 32 ** 3)])
def test_potential_vs_oracle(kind, fsize, n):
    """TVG_CFG_POTENTIAL at larger sizes against the restatement
    (port.walk(potential=True), itself pinned to the reference's golden
    potential): the plain form's Grav_Pot bit for bit, both passes. In FP32
    with the Ewald part both take the separation in double (the reference
    leaves that case undefined)."""
    p, origin, size = make_case(kind, n)
    ft = port.ftype(fsize)
    o = oracle_pipeline(p.pos, p.mass, origin, size, fsize, box=p.box, softening=p.softening,
                        passes=())
    prm = port.WalkParams(gravity=43007.1, softening=p.softening, domain_size=size, boxsize=p.box,
                          open_bh=0.25, open_rel=0.005, use_bh=1, vector_size=64)
    tabs = None
    if p.box > 0:
        fx, fy, fz, fpt = reference_table(fsize)
        tabs = [(t.astype(np.float64) / (p.box * p.box)).astype(ft) for t in (fx, fy, fz)]
        tabs.append((fpt.astype(np.float64) / p.box).astype(ft))

    def oracle_pass(use_bh, last):
        prm.use_bh = use_bh
        _, _, pg = port.walk("gravity", o["pos"], o["mass"], last, o["top"], o["tree"], prm,
                             fsize=fsize, potential=True)
        pot = pg.astype(ft)
        if p.box > 0:
            _, _, pe = port.walk("ewald", o["pos"], o["mass"], last, o["top"], o["tree"], prm, tabs,
                                 fsize=fsize, potential=True)
            pot = (pot.astype(np.float64) + pe).astype(ft)
        return pot

    with make_ctx(p.n, fsize, box=p.box, softening=p.softening, flags=G.CFG_POTENTIAL) as ctx:
        gpu_pipeline(ctx, p.pos, p.mass, origin, size)
        parts = G.WALK_GRAVITY | (G.WALK_EWALD if p.box > 0 else 0)
        if p.box > 0:
            ctx.upload_ewald_table(*reference_table(fsize))
        ctx.zero_accel()
        ctx.walk(G.FORM_PLAIN, use_bh=True, parts=parts)
        bh = ctx.download(G.F_GRAV_POT)["grav_pot"]
        ctx.save_last_accel()
        last = ctx.download(G.F_LAST_ACC)["last_acc_mag"]
        ctx.walk(G.FORM_PLAIN, use_bh=False, parts=parts)
        rel = ctx.download(G.F_GRAV_POT)["grav_pot"]
    for name, got, ref in (("bh", bh, oracle_pass(1, np.zeros(p.n, ft))),
                           ("rel", rel, oracle_pass(0, last.astype(ft)))):
        assert np.array_equal(got, ref), f"{name}: max diff {np.abs(got.astype(float) - ref).max()}"
