"""Build oracle/liboracle.so from oracle/oracle.c (test infrastructure only).

gcc -O2 -fopenmp -ffp-contract=off: float arithmetic is evaluated exactly as written, with
no fused multiply-add, which is the rounding the CUDA library is built for (-fmad=false).
"""
from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SO = HERE / "liboracle.so"


def build(verbose: bool = False) -> Path:
    src = HERE / "oracle.c"
    if SO.exists() and SO.stat().st_mtime >= src.stat().st_mtime:
        return SO
    cmd = ["gcc", "-std=gnu11", "-O2", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
           "-fno-fast-math", "-Wall", "-Wno-unused-function", str(src), "-o", str(SO), "-lm"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return SO


if __name__ == "__main__":
    print(build(verbose=True))
