"""The ctypes mirrors in tandav_b200/gravity.py against the C structs of
include/tandav_gpu.h: a small C program compiled with the system compiler
prints each struct's size and member offsets, which must equal the ctypes
layout (a caller binding the library from C and the Python view must agree
byte for byte)."""
import ctypes as C
import json
import shutil
import subprocess
from pathlib import Path

import pytest

from tandav_b200 import gravity as G

ROOT = Path(__file__).resolve().parents[1]

STRUCTS = [("tvg_config", G.Config), ("tvg_particles", G.Particles),
           ("tvg_timeline_config", G.TimelineConfig), ("tvg_timeline_state", G.TimelineState),
           ("tvg_mlp_train_config", G.MlpTrainConfig),
           ("tvg_snapshot_header", G.SnapshotHeader)]


def _c_layout(tmp_path):
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "tandav_gpu.h"',
             "int main(void) {", '  printf("{");']
    first = True
    for cname, cls in STRUCTS:
        sep = "" if first else ","
        first = False
        lines.append(f'  printf("{sep}\\"{cname}\\": {{\\"size\\": %zu", sizeof({cname}));')
        for field, _ in cls._fields_:
            lines.append(f'  printf(", \\"{field}\\": %zu", offsetof({cname}, {field}));')
        lines.append('  printf("}");')
    lines += ['  printf("}\\n");', "  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    return json.loads(subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout)


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_ctypes_structs_match_the_header(tmp_path):
    got = _c_layout(tmp_path)
    for cname, cls in STRUCTS:
        c = got[cname]
        assert c["size"] == C.sizeof(cls), cname
        for field, _ in cls._fields_:
            assert c[field] == getattr(cls, field).offset, f"{cname}.{field}"


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_topnode_dtype_matches_the_header(tmp_path):
    """gravity.TOPNODE_DTYPE (what tvg_download_tree fills) against
    tvg_topnode: size and the offset of every field."""
    names = {"Key": "key", "Target": "target", "Level": "level", "First_Part": "first_part",
             "Npart": "npart", "Pos": "pos", "Mass": "mass", "CoM": "com", "Dp": "dp"}
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "tandav_gpu.h"',
             "int main(void) {", '  printf("%zu", sizeof(tvg_topnode));']
    for c in names.values():
        lines.append(f'  printf(" %zu", offsetof(tvg_topnode, {c}));')
    lines += ['  printf("\\n");', "  return 0;", "}"]
    src = tmp_path / "top.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "top"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    vals = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True,
                                           text=True).stdout.split()]
    dt = G.TOPNODE_DTYPE
    assert vals[0] == dt.itemsize
    assert vals[1:] == [dt.fields[f][1] for f in names]
