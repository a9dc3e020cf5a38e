"""Build recipe for the oracle (CPU restatement of the Krylov-solve path).

TEST INFRASTRUCTURE: the library built here is the checker and the timed CPU
baseline; the product never links it. Output: oracle/build/liboracle.so.

The reference itself (Fortran 2008 + PSyclone DSL) cannot be compiled in this
environment (no Fortran compiler, no PSyclone), so there is no oracle/_ref.
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "build" / "liboracle.so"

# x86-64-v3 (AVX2 + FMA) so that fma() is one instruction on any recent host;
# -ffp-contract=off keeps every other product and sum unfused.
CFLAGS = ["-O3", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
          "-march=x86-64-v3", "-fno-math-errno"]


def build(force: bool = False) -> Path:
    src = HERE / "oracle.c"
    hdr = HERE / "oracle.h"
    if force or not OUT.exists() or max(src.stat().st_mtime, hdr.stat().st_mtime) > OUT.stat().st_mtime:
        OUT.parent.mkdir(exist_ok=True)
        cmd = ["gcc", *CFLAGS, str(src), "-o", str(OUT), "-lm"]
        print("+", " ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv)
