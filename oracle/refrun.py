"""Run the reference (built by oracle/Makefile into oracle/_ref/) on one input.

Test infrastructure only: this module is the checker's handle on the real
reference program (``ref_harness``, linked against the unmodified reference
sources). It writes the harness input file, runs the binary and parses the
named records it dumps. Nothing in the product imports it.
"""
from __future__ import annotations

import os
import struct
import subprocess
import tempfile
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
REF_DIR = ORACLE_DIR / "_ref"

# struct Tree_Node (src/Gravity/tree.h:23-32) for Float = float / double
TREE_DTYPE = {
    4: np.dtype([("DNext", "<i4"), ("Bitfield", "<u4"), ("DUp", "<i4"), ("Npart", "<i4"),
                 ("Pos", "<f4", 3), ("Mass", "<f4"), ("CoM", "<f4", 3), ("Dp", "<f4", 3)]),
    8: np.dtype([("DNext", "<i4"), ("Bitfield", "<u4"), ("DUp", "<i4"), ("Npart", "<i4"),
                 ("Pos", "<f8", 3), ("Mass", "<f8"), ("CoM", "<f8", 3), ("Dp", "<f8", 3)]),
}
# Top_Tree_Node fields as ref_harness.c dumps them (src/domain.h:40-52)
TOPNODE_DTYPE = np.dtype([("Key", "<u8"), ("Target", "<i4"), ("Level", "<i4"),
                          ("First_Part", "<i4"), ("Npart", "<i4"), ("Pos", "<f4", 3),
                          ("Mass", "<f4"), ("CoM", "<f4", 3), ("Dp", "<f4", 3)])


def harness_path(variant: str) -> Path:
    return REF_DIR / variant / "ref_harness"


def available(variant: str) -> bool:
    return harness_path(variant).exists()


def write_input(path, pos, vel, mass, box=0.0, softening=0.01, flags=3,
                origin=(0.0, 0.0, 0.0), size=1.0):
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    vel = np.ascontiguousarray(vel, dtype=np.float64)
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    n = mass.shape[0]
    with open(path, "wb") as f:
        f.write(b"TVIN")
        f.write(struct.pack("<iq", 1, n))
        f.write(struct.pack("<dd", box, softening))
        f.write(struct.pack("<ddd", *origin))
        f.write(struct.pack("<d", size))
        f.write(struct.pack("<ii", flags, 0))
        f.write(pos.tobytes())
        f.write(vel.tobytes())
        f.write(mass.tobytes())


def read_output(path) -> dict:
    raw = Path(path).read_bytes()
    out, off = {}, 0
    while off < len(raw):
        name = raw[off:off + 16].split(b"\0", 1)[0].decode()
        (nbytes,) = struct.unpack_from("<q", raw, off + 16)
        off += 24
        out[name] = raw[off:off + nbytes]
        off += nbytes
    return out


def keys_u128(buf: bytes) -> np.ndarray:
    """128-bit keys as an (n, 2) uint64 array [hi, lo]."""
    a = np.frombuffer(buf, dtype="<u8").reshape(-1, 2)
    return np.ascontiguousarray(a[:, ::-1])


def run(variant: str, mode: str, pos, vel=None, mass=None, box=0.0, softening=0.01,
        flags=3, origin=(0.0, 0.0, 0.0), size=1.0, threads: int = 1,
        workdir: str | None = None, timeout: float = 3600.0) -> dict:
    """Run ``ref_harness <mode>`` for one particle set and return parsed records."""
    exe = harness_path(variant)
    if not exe.exists():
        raise FileNotFoundError(f"{exe} missing: run `make -C oracle ref`")
    n = np.asarray(pos).shape[1]
    vel = np.zeros((3, n)) if vel is None else vel
    mass = np.full(n, 1.0 / n) if mass is None else mass
    # the reference caches its Ewald table in ./ewald_tables.dat (Gravity/periodic.c:19)
    wd = Path(workdir) if workdir else REF_DIR / variant / "work"
    wd.mkdir(parents=True, exist_ok=True)
    with tempfile.TemporaryDirectory() as td:
        fin, fout = Path(td) / "in.bin", Path(td) / "out.bin"
        write_input(fin, pos, vel, mass, box, softening, flags, origin, size)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        proc = subprocess.run([str(exe), mode, str(fin), str(fout)], cwd=wd, env=env,
                              stdout=subprocess.PIPE, stderr=subprocess.PIPE, timeout=timeout)
        if proc.returncode != 0:
            raise RuntimeError(f"ref_harness failed ({proc.returncode}): "
                               f"{proc.stderr.decode()[-2000:]}{proc.stdout.decode()[-2000:]}")
        rec = read_output(fout)
        snap = Path(str(fout) + "_000")
        snap_bytes = snap.read_bytes() if mode == "snap" and snap.exists() else None
    out = decode(rec, n)
    if snap_bytes is not None:
        out["snapshot"] = snap_bytes       # the file Write_Snapshot wrote
    return out


def read_snapshot(variant: str, path, threads: int = 1, timeout: float = 600.0) -> dict:
    """Run the reference's Read_Snapshot (``ref_harness read``) on a snapshot
    file (or the files path.0, path.1, ...) and return what it loaded."""
    exe = harness_path(variant)
    if not exe.exists():
        raise FileNotFoundError(f"{exe} missing: run `make -C oracle ref`")
    with tempfile.TemporaryDirectory() as td:
        fout = Path(td) / "out.bin"
        env = dict(os.environ, OMP_NUM_THREADS=str(threads))
        proc = subprocess.run([str(exe), "read", str(path), str(fout)], cwd=td, env=env,
                              stdout=subprocess.PIPE, stderr=subprocess.PIPE, timeout=timeout)
        if proc.returncode != 0:
            raise RuntimeError(f"ref_harness read failed ({proc.returncode}): "
                               f"{proc.stderr.decode()[-2000:]}{proc.stdout.decode()[-2000:]}")
        rec = read_output(fout)
    n = struct.unpack("<q", rec["read_n"])[0]
    fsize = struct.unpack("<i", rec["float_size"])[0]
    return dict(n=n, float_size=fsize,
                id=np.frombuffer(rec["read_id"], "<u4").copy(),
                type=np.frombuffer(rec["read_type"], "<i4").copy(),
                pos=np.frombuffer(rec["read_pos"], "<f8").reshape(3, n).copy(),
                vel=np.frombuffer(rec["read_vel"], "<f8").reshape(3, n).copy(),
                mass=np.frombuffer(rec["read_mass"], "<f8").copy(),
                acc0=np.frombuffer(rec["read_acc0"], "<f8").copy(),
                grav_acc=np.frombuffer(rec["read_gacc"], "<f8").reshape(3, n).copy(),
                sim_npart=np.frombuffer(rec["sim_npart"], "<i8").copy(),
                sim_mpart=np.frombuffer(rec["sim_mpart"], "<f8").copy())


def decode(rec: dict, n: int) -> dict:
    out = {}
    fsize = struct.unpack("<i", rec["float_size"])[0] if "float_size" in rec else 4
    for name, buf in rec.items():
        if name in ("std_key", "rev_key"):
            out[name] = keys_u128(buf)
        elif name in ("perm", "id_in"):
            out[name] = np.frombuffer(buf, dtype="<u4").copy()
        elif name == "tree" or name.endswith("_tree"):
            out[name] = np.frombuffer(buf, dtype=TREE_DTYPE[fsize]).copy()
        elif name == "topnodes" or name.endswith("_top"):
            out[name] = np.frombuffer(buf, dtype=TOPNODE_DTYPE).copy()
        elif name == "tree_parent":
            out[name] = np.frombuffer(buf, dtype="<i4").copy()
        elif name == "float_size":
            out[name] = fsize
        elif name.endswith("_acc") or name.endswith("_gacc") or name == "pos":
            out[name] = np.frombuffer(buf, dtype="<f8").reshape(3, n).copy()
        else:
            out[name] = np.frombuffer(buf, dtype="<f8").copy()
    return out
