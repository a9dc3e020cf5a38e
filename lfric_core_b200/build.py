"""In-tree build of the package's native libraries.

liblfx.so          CUDA kernels + C-ABI (include/lfx.h), nvcc for sm_100a only
liblfx_meshgen.so  host-side synthetic-input generator (include/lfx_meshgen.h)

Both land in lfric_core_b200/lib/ so that they travel with the source tree.
"""
from __future__ import annotations

import hashlib
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


def _digest(deps, cmd=()) -> str:
    h = hashlib.sha256()
    for d in sorted(str(x) for x in deps):
        h.update(Path(d).name.encode())
        h.update(Path(d).read_bytes())
    h.update(" ".join(str(c) for c in cmd).encode())
    return h.hexdigest()


def _stamp(target: Path) -> Path:
    return target.with_name(target.name + ".stamp")


def _stale(target: Path, deps, cmd=()) -> bool:
    """True unless `target` exists and was built from sources with these
    exact contents (a digest stamp beside it: copying the tree, which moves
    modification times, does not force a rebuild; editing a source does)."""
    st = _stamp(target)
    if not target.exists() or not st.exists():
        return True
    return st.read_text().strip() != _digest(deps, cmd)


def _mark(target: Path, deps, cmd=()) -> None:
    _stamp(target).write_text(_digest(deps, cmd) + "\n")


def _run(cmd):
    print("+", " ".join(str(c) for c in cmd), flush=True)
    subprocess.run([str(c) for c in cmd], check=True)


def build_meshgen(force: bool = False) -> Path:
    out = LIB / "liblfx_meshgen.so"
    src = CSRC / "meshgen.c"
    deps = [src, INCLUDE / "lfx_meshgen.h"]
    if force or _stale(out, deps):
        LIB.mkdir(exist_ok=True)
        _run(["gcc", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
              f"-I{INCLUDE}", src, "-o", out, "-lm"])
        _mark(out, deps)
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
                _mark(obj, [src] + CU_HEADERS)
            objs.append(obj)
        _run([NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", *objs, "-o", out,
              "-lcudart_static", "-lrt", "-ldl", "-lpthread"])
        _mark(out, CU_SOURCES + CU_HEADERS)
    return out


def build_all(force: bool = False) -> None:
    build_meshgen(force)
    build_lfx(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
