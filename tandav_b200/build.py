"""Builds the in-tree CUDA library tandav_b200/libtandav_gpu.so for sm_100a.

Each .cu file is compiled to an object with nvcc (-gencode
arch=compute_100a,code=sm_100a) and the objects are linked into one shared
library with a plain C ABI (include/tandav_gpu.h). Files whose arithmetic must
round exactly like the reference C code are compiled with -fmad=false.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "libtandav_gpu.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-I", str(ROOT / "include")]
# translation units that replay the reference's rounding order
NO_FMA = {"tvg_walk_plain.cu", "tvg_tree.cu", "tvg_ewald.cu", "tvg_keys.cu", "tvg_integrate.cu",
          "tvg_tree_update.cu"}
# FP32 walks with no parity constraint: denormals flushed (rsqrtf and the
# divisions then need no range fix-up around MUFU)
FTZ = {"tvg_walk_group.cu"}


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _compile(src: Path) -> Path:
    obj = OBJ / (src.stem + ".o")
    deps = ([src] + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.inc"))
            + [ROOT / "include" / "tandav_gpu.h"])
    if obj.exists() and all(obj.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return obj
    flags = list(COMMON)
    if src.name in NO_FMA:
        flags.append("-fmad=false")
    if src.name in FTZ:
        flags.append("-ftz=true")
    cmd = [nvcc(), *ARCH, *flags, "-c", str(src), "-o", str(obj)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{proc.stderr}")
    return obj


def build(verbose: bool = False) -> Path:
    OBJ.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(_compile, sources))
    if LIB.exists() and all(LIB.stat().st_mtime >= o.stat().st_mtime for o in objs):
        return LIB
    cmd = [nvcc(), *ARCH, "-shared", "-Xlinker", "--no-undefined", "-o", str(LIB), *map(str, objs),
           "-lcudart"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"link failed:\n{proc.stderr}")
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(verbose=True)
    sys.exit(0)
