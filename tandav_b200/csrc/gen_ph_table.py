"""Generates tvg_ph_table.inc: the Peano-Hilbert curve of the key kernel as a
finite-state table, two levels per entry.

The curve is the one Peano_Key builds (peano.c:122-276): the Hilbert
transpose of Skilling (2004, AIP Conf. Proc. 707, 381) applied to the three
64-bit integer coordinates, read level by level (level k = bit 63 - k of the
transposed coordinates, X0 the most significant bit of the level's 3-bit
digit; the key holds levels 1..42, level 0 = bit 63 only selects the state
below it). A step of the transpose at bit b changes only bits below b, so the
digit of level k depends on the coordinates' bits at levels 1..k alone, and
the curve is a finite automaton: a state (an orientation of the sub-cube)
maps the octant of the next level, o = x << 2 | y << 1 | z, to the digit of
that level and to the state of the child cube.

This script restates the transpose (Skilling's published steps), discovers
the states by their digit maps over all suffixes of
three levels, checks that the automaton reproduces the transpose on random
64-bit coordinates, and writes a table of 64 entries per state indexed by
the octants of two levels (o1 << 3 | o2):

    entry = (d1 << 3 | d2) | next_state << 6       (uint16)

Run: python tandav_b200/csrc/gen_ph_table.py  (writes the .inc beside it).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

def transpose(x0, x1, x2):
    """Skilling's axes-to-transpose step, Gray encoding and the parity undo,
    on uint64 arrays (all 63 bit steps, b = 63 .. 1)."""
    x0, x1, x2 = (np.array(v, dtype=np.uint64, copy=True) for v in (x0, x1, x2))
    for b in range(63, 0, -1):
        q = np.uint64(1 << b)
        mask = np.uint64((1 << b) - 1)
        x0 = np.where((x0 & q) != 0, x0 ^ mask, x0)
        for xi_name in (1, 2):
            xi = x1 if xi_name == 1 else x2
            hit = (xi & q) != 0
            t = (x0 ^ xi) & mask
            new_x0 = np.where(hit, x0 ^ mask, x0 ^ t)
            new_xi = np.where(hit, xi, xi ^ t)
            x0 = new_x0
            if xi_name == 1:
                x1 = new_xi
            else:
                x2 = new_xi
    x1 = x1 ^ x0
    x2 = x2 ^ x1
    p = x2.copy()
    for s in (1, 2, 4, 8, 16, 32):
        p ^= p >> np.uint64(s)
    above = p ^ x2
    return x0 ^ above, x1 ^ above, x2 ^ above


def level_digits(x0, x1, x2, levels):
    """Digits of the transposed coordinates' bits 63, 62, ..., 64 - levels
    (bit 63 is level 0, above the key's levels 1..42)."""
    t0, t1, t2 = transpose(x0, x1, x2)
    out = np.zeros((len(t0), levels), np.int64)
    for k in range(levels):
        s = np.uint64(63 - k)
        out[:, k] = (((t0 >> s) & np.uint64(1)) << np.uint64(2)
                         | ((t1 >> s) & np.uint64(1)) << np.uint64(1)
                         | ((t2 >> s) & np.uint64(1))).astype(np.int64)
    return out


def coords_of(octs):
    """Coordinates whose bits 63, 62, ... hold the given octants (rows)."""
    octs = np.atleast_2d(np.asarray(octs, np.int64))
    x = [np.zeros(octs.shape[0], np.uint64) for _ in range(3)]
    for k in range(octs.shape[1]):
        s = np.uint64(63 - k)
        o = octs[:, k].astype(np.uint64)
        x[0] |= ((o >> np.uint64(2)) & np.uint64(1)) << s
        x[1] |= ((o >> np.uint64(1)) & np.uint64(1)) << s
        x[2] |= (o & np.uint64(1)) << s
    return x


DEPTH = 3
SUFFIX = np.array(np.meshgrid(*([np.arange(8)] * DEPTH), indexing="ij")).reshape(DEPTH, -1).T


def signature(prefix):
    """Digits of every 3-level suffix below a prefix (the state's behaviour)."""
    rows = np.hstack([np.tile(np.asarray(prefix, np.int64), (len(SUFFIX), 1)), SUFFIX])
    d = level_digits(*coords_of(rows), levels=rows.shape[1])
    return tuple(d[:, len(prefix):].ravel().tolist())


def discover():
    """States and their one-level transitions (digit, next state)."""
    sigs = {}
    prefixes = []
    trans = []
    todo = [()]
    sigs[signature(())] = 0
    prefixes.append(())
    while todo:
        pre = todo.pop(0)
        sid = sigs[signature(pre)]
        row = []
        for o in range(8):
            child = pre + (o,)
            digit = int(level_digits(*coords_of([child]), levels=len(child))[0, -1])
            sg = signature(child)
            if sg not in sigs:
                sigs[sg] = len(prefixes)
                prefixes.append(child)
                todo.append(child)
            row.append((digit, sigs[sg]))
        while len(trans) <= sid:
            trans.append(None)
        trans[sid] = row
    return trans


def check(trans, n=20000, seed=7):
    """The automaton against the transpose on random 64-bit coordinates."""
    rng = np.random.default_rng(seed)
    x = [rng.integers(0, 1 << 64, n, dtype=np.uint64) for _ in range(3)]
    x[0][: n // 2] >>= np.uint64(1)           # half of them below 2^63 in every axis
    x[1][: n // 2] >>= np.uint64(1)
    x[2][: n // 2] >>= np.uint64(1)
    ref = level_digits(*x, levels=43)
    st = np.zeros(n, np.int64)
    tab_d = np.array([[trans[s][o][0] for o in range(8)] for s in range(len(trans))])
    tab_n = np.array([[trans[s][o][1] for o in range(8)] for s in range(len(trans))])
    for k in range(43):
        s = np.uint64(63 - k)
        o = (((x[0] >> s) & np.uint64(1)) << np.uint64(2) | ((x[1] >> s) & np.uint64(1)) << np.uint64(1)
             | ((x[2] >> s) & np.uint64(1))).astype(np.int64)
        d = tab_d[st, o]
        if not np.array_equal(d, ref[:, k]):
            raise SystemExit(f"automaton differs from the transpose at bit {63 - k}")
        st = tab_n[st, o]


def table2(trans):
    """64 entries per state: two levels per lookup."""
    out = []
    for s in range(len(trans)):
        for o1 in range(8):
            d1, s1 = trans[s][o1]
            for o2 in range(8):
                d2, s2 = trans[s1][o2]
                out.append((d1 << 3 | d2) | s2 << 6)
    return out


def main() -> int:
    trans = discover()
    check(trans)
    t2 = table2(trans)
    ns = len(trans)
    lines = [
        "// Generated by gen_ph_table.py: the Peano-Hilbert curve of Peano_Key",
        "// (Skilling's transpose, peano.c:122-276) as a finite-state table, two",
        "// levels per entry. Index: state * 64 + (octant1 << 3 | octant2), octant",
        "// = x << 2 | y << 1 | z of the level's coordinate bits. Entry: the two",
        "// levels' digits (d1 << 3 | d2) | next state << 6. tvg_ph_start: the",
        "// state below bit 63 (level 0, above the key's 42 levels) by its octant.",
        f"#define TVG_PH_STATES {ns}",
        "static __device__ const uint8_t tvg_ph_start[8] = {"
        + ", ".join(str(trans[0][o][1]) for o in range(8)) + "};",
        f"static __device__ const uint16_t tvg_ph_table2[{ns * 64}] = {{",
    ]
    for r in range(0, len(t2), 16):
        lines.append("\t" + ", ".join(f"{v:#06x}" for v in t2[r:r + 16]) + ",")
    lines.append("};")
    dst = Path(__file__).resolve().parent / "tvg_ph_table.inc"
    dst.write_text("\n".join(lines) + "\n")
    print(f"{ns} states, {len(t2)} entries -> {dst}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
