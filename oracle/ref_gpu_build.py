"""Build recipe for oracle/_ref/libref_gpu.so -- the reference's own GPU step on this GPU.

BASELINE INFRASTRUCTURE ONLY.  The product never loads what this script builds.

Compiles, for sm_100a, the reference's CUDA sources on the grid DEM path where they lie in the
checkout -- Kernels/particleKernels.cu, Kernels/rigidBodyKernels.cu,
RigidBodies/UniformGridDEM.cu and WallCollisions.cu (which defines a kernel the second one
launches) -- and oracle/ref_gpu_driver.cu (this repository's host driver of
the reference's step), then links them into ``oracle/_ref/libref_gpu.so``.  Nothing from the
reference is copied: the sources are compiled in place.  Build shims: the empty GL / curand
stand-in headers that oracle/ref_build.py writes to ``oracle/_ref/shim``, ``-include cuda.h``
(the vendored glm 0.9.7 detects CUDA through CUDA_VERSION), and a prelude declaring a
``const float3&`` unary minus (Libs/common/inc/helper_math.h only has ``float3&``, and
RigidBodies/UniformGridDEM.cu negates an rvalue, which MSVC accepted).  CUB comes from this
toolkit.  Without the reference checkout nothing is built.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
LIB = OUT / "libref_gpu.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
SOURCES = ["Kernels/particleKernels.cu", "Kernels/rigidBodyKernels.cu",
           "RigidBodies/UniformGridDEM.cu",
           "WallCollisions.cu"]  # defines CreateIndexKernel, which rigidBodyKernels.cu launches
PRELUDE = """#pragma once
#include <cuda_runtime.h>
inline __host__ __device__ float3 operator-(const float3& a) {
  return make_float3(-a.x, -a.y, -a.z);
}
"""


def reference_root() -> Path:
    return Path(os.environ.get("AR_REFERENCE_ROOT", "/root/reference"))


def build(verbose: bool = False) -> Path | None:
    root = reference_root()
    a = root / "AR_Sim"
    shim = OUT / "shim"
    if not a.is_dir() or not shim.is_dir():
        return None
    objdir = OUT / "gpu_obj"
    objdir.mkdir(parents=True, exist_ok=True)
    prelude = OUT / "ref_gpu_prelude.h"
    prelude.write_text(PRELUDE)
    flags = ["-std=c++14", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-w",
             "-Xcompiler", "-fPIC", "-include", "cuda.h", "-include", str(prelude),
             "-I", str(shim)] + sum((["-I", str(a / d)] for d in
                                     ("BVHSource", "Kernels", "Headers", "RigidBodies",
                                      "Particles")), []) + \
            ["-I", str(root / "Libs" / "common" / "inc"), "-I", str(root / "Libs" / "glm")]
    srcs = [a / s for s in SOURCES] + [HERE / "ref_gpu_driver.cu"]
    newest_src = max(p.stat().st_mtime for p in srcs + [Path(__file__)])
    if LIB.exists() and LIB.stat().st_mtime >= newest_src:
        return LIB

    def compile_one(src: Path) -> Path:
        obj = objdir / (src.stem + ".o")
        cmd = [NVCC, *flags, "-c", str(src), "-o", str(obj)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr[-4000:]}")
        return obj

    with cf.ThreadPoolExecutor(max_workers=4) as ex:
        objs = list(ex.map(compile_one, srcs))
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(LIB),
           *map(str, objs), "-lcudart", "-Xlinker", "--no-undefined"]
    subprocess.run(cmd, check=True, capture_output=not verbose)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv))
