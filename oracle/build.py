"""Build recipe for the oracle (CPU restatement of the Krylov-solve path).

TEST INFRASTRUCTURE: the library built here is the checker and the timed CPU
baseline; the product never links it. Output: oracle/build/liboracle.so.

The reference itself (Fortran 2008 + PSyclone DSL) cannot be compiled in this
environment (no Fortran compiler, no PSyclone), so there is no oracle/_ref.
"""
from __future__ import annotations

import hashlib
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "build" / "liboracle.so"

# x86-64-v3 (AVX2 + FMA) so that fma() is one instruction on any recent host;
# -ffp-contract=off keeps every other product and sum unfused.
CFLAGS = ["-O3", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
          "-march=x86-64-v3", "-fno-math-errno"]


def _digest() -> str:
    h = hashlib.sha256()
    for f in ("oracle.c", "oracle.h"):
        h.update((HERE / f).read_bytes())
    h.update(" ".join(CFLAGS).encode())
    return h.hexdigest()


def build(force: bool = False) -> Path:
    """Compiles the oracle unless the library beside its digest stamp was
    built from these exact sources."""
    stamp = OUT.with_name(OUT.name + ".stamp")
    dg = _digest()
    if force or not OUT.exists() or not stamp.exists() or stamp.read_text().strip() != dg:
        OUT.parent.mkdir(exist_ok=True)
        cmd = ["gcc", *CFLAGS, str(HERE / "oracle.c"), "-o", str(OUT), "-lm"]
        print("+", " ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        stamp.write_text(dg + "\n")
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv)
