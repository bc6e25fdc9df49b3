"""The key kernel's Peano-Hilbert state table (tandav_b200/csrc/tvg_ph_table.inc)
against the oracle's keys, which are pinned bit for bit to the reference's
Peano_Key / Reversed_Peano_Key (peano.c:122-276).

The table-driven walk of k_ph_keys (tvg_keys.cu) is restated here in numpy,
step for step: the octants of levels 1..42 from the scaled integer
coordinates, the start state from bit 63, 21 lookups of two levels each, and
the placement of the digits in the standard and reversed 128-bit keys. Both
key orders must equal the oracle's on the reference's own 4^3 grid, on the
corner and near-one points and on random positions in FP32 and FP64. The
generated file must also be what the generator writes now."""
import re
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

import port

ROOT = Path(__file__).resolve().parents[1]
INC = ROOT / "tandav_b200" / "csrc" / "tvg_ph_table.inc"
GEN = ROOT / "tandav_b200" / "csrc" / "gen_ph_table.py"
U = np.uint64


def load_table():
    text = INC.read_text()
    start = [int(v) for v in re.search(r"tvg_ph_start\[8\] = \{([^}]*)\}", text).group(1).split(",")]
    body = re.search(r"tvg_ph_table2\[\d+\] = \{([^}]*)\}", text, re.S).group(1)
    tab = [int(v, 16) for v in body.replace("\n", " ").split(",") if v.strip()]
    return np.array(start, np.int64), np.array(tab, np.int64)


def spread3(v):
    v = v & U(0x1FFFFF)
    v = (v | (v << U(32))) & U(0x1F00000000FFFF)
    v = (v | (v << U(16))) & U(0x1F0000FF0000FF)
    v = (v | (v << U(8))) & U(0x100F00F00F00F00F)
    v = (v | (v << U(4))) & U(0x10C30C30C30C30C3)
    v = (v | (v << U(2))) & U(0x1249249249249249)
    return v


def table_keys(pos, origin, size, fsize):
    """k_ph_keys restated: (std, rev) as (n, 2) uint64 [hi, lo]."""
    start, tab = load_table()
    ft = np.float32 if fsize == 4 else np.float64
    fac = float(1 << 63) / size
    s = [(pos[k].astype(ft).astype(np.float64) - origin[k]) * fac for k in range(3)]
    x0, x1, x2 = (v.astype(np.uint64) for v in s)
    mh = (spread3(x0 >> U(42)) << U(2)) | (spread3(x1 >> U(42)) << U(1)) | spread3(x2 >> U(42))
    ml = (spread3(x0 >> U(21)) << U(2)) | (spread3(x1 >> U(21)) << U(1)) | spread3(x2 >> U(21))
    st = start[((x0 >> U(63)) << U(2) | (x1 >> U(63)) << U(1) | (x2 >> U(63))).astype(np.int64)]
    n = len(x0)
    dh = np.zeros(n, np.uint64)
    dl = np.zeros(n, np.uint64)
    rh = np.zeros(n, np.uint64)
    rl = np.zeros(n, np.uint64)

    def swap(e):
        return (((e >> 3) & 7) | ((e & 7) << 3)).astype(np.uint64)

    for j in range(10):
        e = tab[st * 64 + ((mh >> U(57 - 6 * j)) & U(63)).astype(np.int64)]
        st = e >> 6
        dh |= (e & 63).astype(np.uint64) << U(57 - 6 * j)
        rh |= swap(e) << U(6 * j)
    e = tab[st * 64 + (((mh & U(7)) << U(3)) | ((ml >> U(60)) & U(7))).astype(np.int64)]
    st = e >> 6
    dh |= ((e >> 3) & 7).astype(np.uint64)
    dl |= (e & 7).astype(np.uint64) << U(60)
    rh |= ((e >> 3) & 7).astype(np.uint64) << U(60)
    rl |= (e & 7).astype(np.uint64)
    for j in range(10):
        e = tab[st * 64 + ((ml >> U(54 - 6 * j)) & U(63)).astype(np.int64)]
        st = e >> 6
        dl |= (e & 63).astype(np.uint64) << U(54 - 6 * j)
        rl |= swap(e) << U(3 + 6 * j)
    std = np.stack([(dh << U(1)) | (dl >> U(62)), dl << U(2)], axis=1)
    rev = np.stack([(rh >> U(61)) | (rl << U(2)), rh << U(3)], axis=1)
    return std, rev


def test_generated_table_is_current(tmp_path):
    """Re-running the generator (which checks its automaton against the
    transpose on random coordinates) reproduces the committed table."""
    before = INC.read_text()
    out = subprocess.run([sys.executable, str(GEN)], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    assert INC.read_text() == before


@pytest.mark.parametrize("fsize", [4, 8])
def test_table_keys_on_the_reference_grid(golden_dir, fsize):
    g = np.load(golden_dir / "keys_grid.npz")
    std, rev = table_keys(g["pos"], (0.0, 0.0, 0.0), 1.0, fsize)
    variant = "iso_f32" if fsize == 4 else "iso_f64"
    assert np.array_equal(std, g[f"{variant}_std"])
    assert np.array_equal(rev, g[f"{variant}_rev"])


@pytest.mark.parametrize("fsize", [4, 8])
def test_table_keys_match_the_oracle(fsize):
    rng = np.random.default_rng(11 + fsize)
    n = 200_000
    origin = np.array([-3.5, 2.0, 10.25])
    size = 7.75
    pos = origin[:, None] + size * rng.random((3, n))
    # corners, the far faces and points just below them
    edge = np.array([0.0, 1.0 - 1e-10, 0.5, 1.0 - 2.0 ** -40, 2.0 ** -43])
    g = np.array(np.meshgrid(edge, edge, edge, indexing="ij")).reshape(3, -1)
    pos = np.hstack([pos, origin[:, None] + size * g])
    ft = np.float32 if fsize == 4 else np.float64
    pos = pos.astype(ft)
    # keep every coordinate inside [origin, origin + size) after rounding
    pos = np.minimum(np.maximum(pos, origin[:, None].astype(ft)),
                     np.nextafter((origin + size)[:, None].astype(ft), ft(-np.inf)))
    std_t, rev_t = table_keys(pos, origin, size, fsize)
    std_o, rev_o = port.peano_keys(pos, origin, size, fsize)
    assert np.array_equal(std_t, std_o)
    assert np.array_equal(rev_t, rev_o)


def test_table_keys_above_the_domain_match_the_oracle():
    """Coordinates up to twice the domain size (bit 63 of the scaled integer
    set): the start state below bit 63 keeps the keys equal to the
    transpose's."""
    rng = np.random.default_rng(5)
    n = 50_000
    pos = 1.999 * rng.random((3, n))
    std_t, rev_t = table_keys(pos, (0.0, 0.0, 0.0), 1.0, 8)
    std_o, rev_o = port.peano_keys(pos, (0.0, 0.0, 0.0), 1.0, 8)
    assert np.array_equal(std_t, std_o)
    assert np.array_equal(rev_t, rev_o)
