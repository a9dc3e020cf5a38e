"""In-tree build of the package's native libraries.

liblfx.so          CUDA kernels + C-ABI (include/lfx.h), nvcc for sm_100a only
liblfx_meshgen.so  host-side synthetic-input generator (include/lfx_meshgen.h)

Both land in lfric_core_b200/lib/ so that they travel with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "lib"
INCLUDE = ROOT / "include"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = sorted(CSRC.glob("*.cu"))
CU_HEADERS = sorted(CSRC.glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd):
    print("+", " ".join(str(c) for c in cmd), flush=True)
    subprocess.run([str(c) for c in cmd], check=True)


def build_meshgen(force: bool = False) -> Path:
    out = LIB / "liblfx_meshgen.so"
    src = CSRC / "meshgen.c"
    if force or _stale(out, [src, INCLUDE / "lfx_meshgen.h"]):
        LIB.mkdir(exist_ok=True)
        _run(["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
              f"-I{INCLUDE}", src, "-o", out, "-lm"])
    return out


def build_lfx(force: bool = False) -> Path:
    out = LIB / "liblfx.so"
    if force or _stale(out, CU_SOURCES + CU_HEADERS):
        LIB.mkdir(exist_ok=True)
        objs = []
        obj_dir = PKG / "_build"
        obj_dir.mkdir(exist_ok=True)
        for src in CU_SOURCES:
            obj = obj_dir / (src.stem + ".o")
            if force or _stale(obj, [src] + CU_HEADERS):
                # -fmad=false (device) and -ffp-contract=off (host): only the
                # explicit fma() calls in the sources are fused, so FP64 results
                # match the CPU oracle bit for bit.
                _run([NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-fmad=false", "--extended-lambda",
                      "-Xcompiler", "-fPIC,-ffp-contract=off",
                      "-Xptxas", "-v" if os.environ.get("LFX_PTXAS_V") else "-O3",
                      f"-I{INCLUDE}", f"-I{CSRC}", "-c", src, "-o", obj])
            objs.append(obj)
        _run([NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", *objs, "-o", out,
              "-lcudart_static", "-lrt", "-ldl", "-lpthread"])
    return out


def build_all(force: bool = False) -> None:
    build_meshgen(force)
    build_lfx(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
