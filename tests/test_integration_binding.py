"""The reference-side binding shown in INTEGRATION.md compiles against the
reference's own headers, and every library function it calls is exported by
libtandav_gpu.so with a prototype from include/tandav_gpu.h.

The C blocks of INTEGRATION.md that define functions are put together as one
translation unit (src/Gravity/gpu_gravity.c in a GPU build) and compiled with
the flags and the generated config.h of the oracle's reference builds
(oracle/Makefile), isolated and periodic. Implicit declarations, pointer
type mismatches and conflicting prototypes are errors. No GPU is used.
"""
import os
import re
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
REF = Path(os.environ.get("TANDAV_REFERENCE", "/root/reference"))
LIB = ROOT / "tandav_b200" / "libtandav_gpu.so"


def binding_source():
    text = (ROOT / "INTEGRATION.md").read_text()
    blocks = re.findall(r"```c\n(.*?)```", text, flags=re.S)
    # whole functions only (fragments of reference functions start indented)
    units = [b for b in blocks if b and not b[0].isspace()]
    assert len(units) >= 3
    return "\n".join(units)


@pytest.mark.parametrize("variant", ["iso_f64", "per_f32"])
def test_integration_binding_compiles_against_the_reference(tmp_path, variant):
    if not (REF / "src" / "includes.h").exists():
        pytest.skip("reference sources not present")
    cfg = ROOT / "oracle" / "_ref" / variant / "config.h"
    if not cfg.exists() or not LIB.exists():
        pytest.skip("oracle reference build or library missing")
    src = tmp_path / "gpu_gravity.c"
    src.write_text(binding_source())
    obj = tmp_path / "gpu_gravity.o"
    cmd = ["gcc", "-std=gnu11", "-fopenmp", "-fcommon", "-include", "float.h", "-include",
           "stddef.h", "-Werror=implicit-function-declaration", "-Werror=incompatible-pointer-types",
           "-Werror=int-conversion", "-Werror=return-type", "-fPIC",
           f"-I{cfg.parent}", f"-I{ROOT / 'oracle' / 'shim'}", f"-I{REF / 'src'}",
           f"-I{REF / 'src' / 'Gravity'}", f"-I{ROOT / 'include'}", "-c", str(src), "-o", str(obj)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    assert proc.returncode == 0, proc.stderr[-4000:]
    # every tvg_ symbol the binding calls is exported by the library
    nm = shutil.which("nm")
    used = subprocess.run([nm, "-u", str(obj)], capture_output=True, text=True, check=True).stdout
    used = {ln.split()[-1] for ln in used.splitlines() if ln.split() and ln.split()[-1].startswith("tvg_")}
    exported = subprocess.run([nm, "-D", "--defined-only", str(LIB)], capture_output=True, text=True,
                              check=True).stdout
    exported = {ln.split()[-1] for ln in exported.splitlines() if ln.split()}
    assert used, "the binding calls no library function"
    assert used <= exported, sorted(used - exported)
    # and the object links against the library (undefined reference symbols
    # are the reference's own, resolved when it links its other objects)
    so = tmp_path / "libbinding.so"
    link = subprocess.run(["gcc", "-shared", "-o", str(so), str(obj), f"-L{LIB.parent}", "-ltandav_gpu"],
                          capture_output=True, text=True)
    assert link.returncode == 0, link.stderr[-2000:]
