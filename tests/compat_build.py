"""Build recipe for tests/_compat/libcompat_driver.so: include/arsim_compat.hpp (the C++ shim
with the reference's wrapper signatures) compiled against the reference's own declaration
headers by tests/compat_driver.cpp, and linked against libarsim.so.

The reference's headers (SimParams, AABB, glm) exist only where the reference checkout is
(``AR_REFERENCE_ROOT``, default ``/root/reference``), so the library is built there, by
``__graft_entry__.build()``, and the built file is what the GPU tests load.  Without the
checkout nothing is built and the shim's GPU test is skipped.
"""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
OUT = HERE / "_compat"
LIB = OUT / "libcompat_driver.so"
STUBS = ROOT / "oracle" / "_ref" / "shim"  # empty GL / curand stand-in headers


def reference_root() -> Path:
    return Path(os.environ.get("AR_REFERENCE_ROOT", "/root/reference"))


def build() -> Path | None:
    ref = reference_root()
    a = ref / "AR_Sim"
    arsim = ROOT / "diploma_thesis_b200" / "libarsim.so"
    if not a.is_dir() or not STUBS.is_dir() or not arsim.exists():
        return None
    OUT.mkdir(exist_ok=True)
    src = HERE / "compat_driver.cpp"
    deps = [src, ROOT / "include" / "arsim_compat.hpp", ROOT / "include" / "arsim.h", arsim]
    if LIB.exists() and LIB.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return LIB
    cmd = ["g++", "-std=c++14", "-O2", "-fPIC", "-shared", "-w",
           "-I", str(STUBS), "-I", "/usr/local/cuda/include", "-I", str(ROOT / "include"),
           "-I", str(a / "Kernels"), "-I", str(a / "BVHSource"), "-I", str(a / "RigidBodies"),
           "-I", str(a / "Particles"), "-I", str(ref / "Libs" / "common" / "inc"),
           "-I", str(ref / "Libs" / "glm"),
           str(src), "-o", str(LIB), str(arsim), "-L/usr/local/cuda/lib64", "-lcudart",
           "-Wl,-rpath,$ORIGIN/../../diploma_thesis_b200"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compat driver build failed:\n{r.stderr[-4000:]}")
    return LIB


if __name__ == "__main__":
    print(build())
