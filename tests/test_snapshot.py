"""Snapshot output (Write_Snapshot, src/IO/write_snapshot.c:13-328): the
library's writer against the file the reference's own Write_Snapshot writes
for the same particles (the reference harness, mode "snap", which also sets
Acc[k] = (k+1) Pos[k], Grav_Acc[k] = (k+2) Vel[k] and Grav_Pot = Pos[0] -
3 Mass so that every block carries distinct data).

Byte for byte, except the header's 64 fill and padding bytes (the reference
leaves them unset) and, without COMOVING, Redshift (also unset there)."""
import ctypes as C
import struct

import numpy as np
import pytest

from oracle import refrun
from tandav_b200 import gravity as G

HEAD = 20            # label record (16 bytes) + the record marker before the header


def _blocks(buf: bytes):
    """Format-2 blocks as (label, payload) with every marker checked."""
    out, off = [], 0
    while off < len(buf):
        m0, label, size8, m1 = struct.unpack_from("<I4sII", buf, off)
        assert (m0, m1) == (8, 8), off
        off += 16
        (a,) = struct.unpack_from("<I", buf, off)
        assert a + 8 == size8, label
        data = buf[off + 4:off + 4 + a]
        (b,) = struct.unpack_from("<I", buf, off + 4 + a)
        assert b == a, label
        out.append((label.decode(), data))
        off += 8 + a
    return out


def _particles(n, box, seed):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0, box, (3, n))
    vel = rng.normal(0, 30.0, (3, n))
    mass = rng.uniform(0.5, 1.5, n) / n
    return pos, vel, mass


def _fields(pos, vel, mass, ft, with_pot):
    k = np.arange(1, 4)[:, None]
    out = dict(pos=pos.astype(ft), vel=vel.astype(ft), ids=np.arange(pos.shape[1], dtype=np.uint32),
               mass=mass.astype(ft), acc=(k * pos).astype(ft), grav_acc=((k + 1) * vel).astype(ft))
    if with_pot:
        out["grav_pot"] = (pos[0] - 3 * mass).astype(ft)
    return out


VARIANTS = [("perc_f32", True, False), ("per_f64", False, False), ("per_f64_pot", False, True),
            ("iso_f32", False, False)]


@pytest.mark.parametrize("variant,comoving,with_pot", VARIANTS)
def test_snapshot_matches_reference_write_snapshot(tmp_path, variant, comoving, with_pot):
    if not refrun.available(variant):
        pytest.skip(f"oracle/_ref/{variant} not built")
    n, box, time = 777, 100.0, 0.02
    pos, vel, mass = _particles(n, box, seed=len(variant))
    ref = refrun.run(variant, "snap", pos, vel, mass, box=box, size=time)
    fb = ref["float_size"]
    ft = np.float32 if fb == 4 else np.float64
    om0, oml, hub = ref["cosmo"]
    h = G.snapshot_header(n, time, box, om0, oml, hub, comoving=comoving)
    f = _fields(pos, vel, mass, ft, with_pot)
    path = tmp_path / "snap_000"
    G.write_snapshot_host(path, h, f["pos"], f["vel"], f["ids"], f["mass"], acc=f["acc"],
                          grav_acc=f["grav_acc"], grav_pot=f.get("grav_pot"))
    ours, theirs = path.read_bytes(), ref["snapshot"]
    labels = ["HEAD", "POS ", "VEL ", "ID  ", "MASS", "ACC ", "GACC"] + (["GPOT"] if with_pot else [])
    assert [b[0] for b in _blocks(theirs)] == labels
    assert [b[0] for b in _blocks(ours)] == labels
    assert len(ours) == len(theirs)
    mask = np.ones(len(ours), bool)
    mask[HEAD + 192:HEAD + 256] = False
    if not comoving:
        mask[HEAD + 80:HEAD + 88] = False
    a, b = np.frombuffer(ours, np.uint8), np.frombuffer(theirs, np.uint8)
    bad = np.flatnonzero((a != b) & mask)
    assert bad.size == 0, f"{bad.size} bytes differ, first at {bad[:8]}"
    # the ACC block is one component, Acc[0], as the reference declares it
    acc_block = dict(_blocks(ours))["ACC "]
    np.testing.assert_array_equal(np.frombuffer(acc_block, ft), f["acc"][0])


def test_snapshot_header_fields(tmp_path):
    """Per-type counts, the 64-bit total split into Nall and Nall_High_Word,
    Massarr, and zero fill; an empty snapshot still has every block."""
    h = G.snapshot_header([0, 0, 0, 0, 0, 0], 0.5, 1000.0, 0.3, 0.7, 0.68,
                          nall=[0, 5_000_000_000, 0, 0, 0, 3], massarr=[0, 2.5, 0, 0, 0, 0],
                          num_files=4)
    z = np.zeros((3, 0))
    path = tmp_path / "empty"
    G.write_snapshot_host(path, h, z, z, np.zeros(0, np.uint32), np.zeros(0))
    blocks = _blocks(path.read_bytes())
    assert [b[0] for b in blocks] == ["HEAD", "POS ", "VEL ", "ID  ", "MASS"]
    assert all(len(b[1]) == 0 for b in blocks[1:])
    head = blocks[0][1]
    assert len(head) == 256
    assert struct.unpack_from("<6I", head, 0) == (0,) * 6
    assert struct.unpack_from("<6d", head, 24) == (0, 2.5, 0, 0, 0, 0)
    assert struct.unpack_from("<dd", head, 72) == (0.5, 1.0)
    assert struct.unpack_from("<6I", head, 96) == (0, 5_000_000_000 & 0xFFFFFFFF, 0, 0, 0, 3)
    assert struct.unpack_from("<6I", head, 168) == (0, 5_000_000_000 >> 32, 0, 0, 0, 0)
    assert struct.unpack_from("<ii", head, 88) == (0, 0)                  # Sfr, Feedback
    assert struct.unpack_from("<ii", head, 120) == (0, 4)                 # Cooling, Num_Files
    assert struct.unpack_from("<4d", head, 128) == (1000.0, 0.3, 0.7, 0.68)
    assert struct.unpack_from("<ii", head, 160) == (0, 0)                 # Age, Metals
    assert head[192:] == bytes(64)


def test_snapshot_rejects_bad_requests(tmp_path):
    """A requested block whose array is NULL, a Float width other than 4/8,
    and an unwritable path are errors (TVG_E_BADINPUT), not crashes."""
    lib = G.lib()
    n = 8
    pos = np.zeros((3, n), np.float32)
    ids = np.arange(n, dtype=np.uint32)
    mass = np.ones(n, np.float32)
    p = G.Particles()
    for k in range(3):
        p.pos[k] = p.vel[k] = pos[k].ctypes.data
    p.id, p.mass = ids.ctypes.data, mass.ctypes.data
    h = G.snapshot_header(n, 1.0, 1.0)

    def call(path, fb, blocks):
        return lib.tvg_write_snapshot_host(str(path).encode(), C.byref(h), C.c_int64(n),
                                           C.c_int32(fb), C.byref(p), C.c_uint32(blocks))

    assert call(tmp_path / "ok", 4, 0) == G.TVG_OK
    assert call(tmp_path / "gacc", 4, G.SNAP_GACC) == 5
    assert call(tmp_path / "pot", 4, G.SNAP_GPOT) == 5
    assert call(tmp_path / "fb", 2, 0) == 5
    assert call(tmp_path / "no" / "such" / "dir", 4, 0) == 5


def test_snapshot_many_particles_matches_numpy_rendering(tmp_path):
    """200,001 particles (the writer interleaves in chunks of 65,536, the last
    one ragged) against the format rendered with numpy: label record, record
    markers, components interleaved per particle."""
    n = 200001
    rng = np.random.default_rng(1)
    pos, vel, gacc = (rng.random((3, n)).astype(np.float32) for _ in range(3))
    ids = np.arange(n, dtype=np.uint32)
    mass = rng.random(n).astype(np.float32)
    h = G.snapshot_header(n, 0.5, 10.0)
    path = tmp_path / "big"
    G.write_snapshot_host(path, h, pos, vel, ids, mass, grav_acc=gacc)
    got = path.read_bytes()

    def rec(label, data):
        return (struct.pack("<I4sII", 8, label, len(data) + 8, 8) + struct.pack("<I", len(data))
                + data + struct.pack("<I", len(data)))

    want = (got[:HEAD + 256 + 4] + rec(b"POS ", pos.T.tobytes()) + rec(b"VEL ", vel.T.tobytes())
            + rec(b"ID  ", ids.tobytes()) + rec(b"MASS", mass.tobytes())
            + rec(b"GACC", gacc.T.tobytes()))
    assert got == want


def _write_typed(base, fsize, files, massarr, rng):
    """Snapshot files holding particles of types 1 and 4 (`files`: their
    counts per file); IDs follow the reference's type ranges (type 1 takes
    [0, n1), type 4 the next n4), shuffled. One file is `base` itself, more
    are base.0, base.1, ... Returns the particles in file order."""
    ft = np.float32 if fsize == 4 else np.float64
    n1, n4 = sum(a for a, _ in files), sum(b for _, b in files)
    id1, id4 = rng.permutation(n1), n1 + rng.permutation(n4)
    nall = [0, n1, 0, 0, n4, 0]
    parts = []
    o1 = o4 = 0
    for i, (a, b) in enumerate(files):
        m = a + b
        pos = rng.uniform(0, 100.0, (3, m)).astype(ft)
        vel = rng.normal(0, 30.0, (3, m)).astype(ft)
        mass = rng.uniform(0.5, 1.5, m).astype(ft)
        gacc = rng.normal(0, 1.0, (3, m)).astype(ft)
        ids = np.concatenate([id1[o1:o1 + a], id4[o4:o4 + b]]).astype(np.uint32)
        o1, o4 = o1 + a, o4 + b
        h = G.snapshot_header([0, a, 0, 0, b, 0], 0.1, 100.0, nall=nall, massarr=massarr,
                              num_files=len(files))
        path = base if len(files) == 1 else f"{base}.{i}"
        G.write_snapshot_host(path, h, pos, vel, ids, mass, grav_acc=gacc)
        parts.append(dict(n1=a, pos=pos, vel=vel, mass=mass, id=ids, grav_acc=gacc))
    return parts


@pytest.mark.parametrize("variant", ["perc_f32", "per_f64"])
@pytest.mark.parametrize("header_mass", [False, True])
def test_reader_matches_reference_read_snapshot(tmp_path, variant, header_mass):
    """tvg_read_snapshot_host against the reference's own Read_Snapshot on a
    two-type snapshot: the same particles in the same order (type sections),
    types from the ID ranges, and with a header mass for type 1 every mass
    from the header (type 4 gets 0 there, as the reference does)."""
    if not refrun.available(variant):
        pytest.skip(f"oracle/_ref/{variant} not built")
    fsize = 4 if variant.endswith("f32") else 8
    massarr = [0, 2.5, 0, 0, 0, 0] if header_mass else [0] * 6
    base = tmp_path / "ics"
    _write_typed(base, fsize, [(190, 80)], massarr, np.random.default_rng(11))
    ref = refrun.read_snapshot(variant, base)
    got = G.read_snapshot(base, fsize)
    assert got["n"] == ref["n"] == 270 and got["num_files"] == 1
    np.testing.assert_array_equal(got["id"], ref["id"])
    np.testing.assert_array_equal(got["type"], ref["type"])
    for k in ("pos", "vel", "mass", "grav_acc"):
        np.testing.assert_array_equal(got[k].astype(np.float64), ref[k], err_msg=k)
    assert list(np.unique(got["type"])) == [1, 4]
    if header_mass:
        assert set(np.unique(got["mass"][got["type"] == 1])) == {2.5}
        assert set(np.unique(got["mass"][got["type"] == 4])) == {0.0}


@pytest.mark.parametrize("header_mass", [False, True])
def test_reader_split_snapshot(tmp_path, header_mass):
    """A snapshot in two files (base.0, base.1; find_files naming) reads as
    Reallocate_P arranges it: the type-1 particles of file 0, then of file 1,
    then the type-4 particles of both. The reference itself cannot read a
    split snapshot here: read_file builds the name with sprintf(filename,
    "%s.%i", filename, ...), whose source and destination overlap."""
    files = [(120, 30), (70, 50)]
    massarr = [0, 2.5, 0, 0, 0, 0] if header_mass else [0] * 6
    base = tmp_path / "ics"
    parts = _write_typed(base, 4, files, massarr, np.random.default_rng(5))
    got = G.read_snapshot(base, 4)
    assert got["n"] == 270 and got["num_files"] == 2

    def arranged(key):
        a = [p[key][..., :p["n1"]] for p in parts] + [p[key][..., p["n1"]:] for p in parts]
        return np.concatenate(a, axis=-1)

    for k in ("pos", "vel", "id", "grav_acc"):
        np.testing.assert_array_equal(got[k], arranged(k), err_msg=k)
    np.testing.assert_array_equal(got["type"], np.repeat([1, 4], [190, 80]))
    if header_mass:
        np.testing.assert_array_equal(got["mass"], np.repeat(np.float32([2.5, 0]), [190, 80]))
    else:
        np.testing.assert_array_equal(got["mass"], arranged("mass"))


def test_reader_round_trip_and_byte_order(tmp_path):
    """What the writer wrote reads back unchanged, also from a copy of the file
    with every record swapped to the other byte order; missing required
    blocks and a Float width that disagrees with the block sizes are errors."""
    n = 500
    rng = np.random.default_rng(2)
    pos, vel, gacc = (rng.random((3, n)) for _ in range(3))
    ids = rng.permutation(n).astype(np.uint32)
    mass = rng.random(n)
    h = G.snapshot_header(n, 0.25, 1.0)
    path = tmp_path / "s"
    G.write_snapshot_host(path, h, pos, vel, ids, mass, grav_acc=gacc)
    got = G.read_snapshot(path, 8)
    for k, v in (("pos", pos), ("vel", vel), ("id", ids), ("mass", mass), ("grav_acc", gacc)):
        np.testing.assert_array_equal(got[k], v, err_msg=k)
    assert got["blocks"] == G.SNAP_MASS | G.SNAP_GACC and got["header"].time == 0.25
    # the same file in big-endian byte order
    swapped = bytearray()
    for label, data in _blocks(path.read_bytes()):
        word = 8
        if label == "HEAD":
            a = np.frombuffer(data, np.uint8).copy()
            for lo, hi, w in ((0, 24, 4), (24, 88, 8), (88, 128, 4), (128, 160, 8), (160, 192, 4)):
                a[lo:hi] = a[lo:hi].reshape(-1, w)[:, ::-1].reshape(-1)
            payload = a.tobytes()
        else:
            w = 4 if label == "ID  " else word
            payload = np.frombuffer(data, np.uint8).reshape(-1, w)[:, ::-1].tobytes()
        swapped += struct.pack(">I4sII", 8, label.encode(), len(payload) + 8, 8)
        swapped += struct.pack(">I", len(payload)) + payload + struct.pack(">I", len(payload))
    (tmp_path / "be").write_bytes(bytes(swapped))
    got_be = G.read_snapshot(tmp_path / "be", 8)
    for k in ("pos", "vel", "id", "mass", "grav_acc"):
        np.testing.assert_array_equal(got_be[k], got[k], err_msg=k)
    # FP64 blocks read as FP32: the sizes disagree
    with pytest.raises(G.TvgError):
        G.read_snapshot(path, 4)
    # a file without VEL
    raw = b"".join(struct.pack("<I4sII", 8, lab.encode(), len(d) + 8, 8) + struct.pack("<I", len(d))
                   + d + struct.pack("<I", len(d))
                   for lab, d in _blocks(path.read_bytes()) if lab != "VEL ")
    (tmp_path / "novel").write_bytes(raw)
    with pytest.raises(G.TvgError):
        G.read_snapshot(tmp_path / "novel", 8)
