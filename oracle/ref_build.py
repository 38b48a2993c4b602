"""Build recipe for oracle/_ref/libref_cpu.so -- the reference's own kernel bodies on the CPU.

TEST INFRASTRUCTURE ONLY (oracle).  The product never loads what this script builds.

AR_Sim's hot path is CUDA.  Its per-particle and per-body kernel bodies are plain C++
apart from a handful of device intrinsics, so this recipe:

1. copies the exact line ranges that hold the hot-path device functions and kernels out
   of the reference checkout into ``oracle/_ref/extracted.inc`` (git-ignored, never
   committed), each range preceded by a ``#line`` directive so compiler messages point
   at the reference file and line;
2. writes four empty stand-in headers for the graphics / curand includes the reference
   headers pull in (no GL or curand call sits in the extracted code);
3. compiles ``oracle/ref_cpu_driver.cpp`` (this repository's own host driver, which
   launches every extracted kernel body over an emulated grid in OpenMP loops) together
   with the extracted code and the reference's vendored headers (helper_math.h, glm
   0.9.7, BVHAuxiliary.cuh, BVHSoAKernels.cu) into ``oracle/_ref/libref_cpu.so``.

The reference is located through ``AR_REFERENCE_ROOT`` (default ``/root/reference``).
When it is absent the build is skipped and callers fall back to the committed golden
fixtures under ``tests/golden/``.

Only the line ranges in ``RANGES`` are used; each is checked against the text expected at
its first line so that a different reference revision fails loudly instead of compiling
the wrong code.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"

# (file relative to AR_Sim/, first line, last line, text the first line must contain)
RANGES = [
    ("BVHSource/BVHkernels.cu", 646, 716, "Expands a 10-bit integer"),          # expandBits, morton3D, generateMortonCodes x2
    ("Kernels/particleKernels.cu", 50, 128, "struct integrate_functor"),       # free-particle integrate
    ("Kernels/particleKernels.cu", 150, 189, "calculate position in uniform grid"),  # calcGridPos, calcGridHash, calcHashD
    ("Kernels/particleKernels.cu", 260, 406, "collide two spheres using DEM"),   # collideSpheres, collideCell, collideD
    ("RigidBodies/UniformGridDEM.cu", 24, 204, "calculate position in uniform grid"),  # DEM grid collide cell + kernel
    ("RigidBodies/UniformGridDEM.cu", 243, 377, "__device__"),                    # AR static-scene DEM cell + kernel
    ("RigidBodies/UniformGridDEM.cu", 420, 460, "Now apply total impulse"),      # CombineReducedImpulses
    ("Kernels/rigidBodyKernels.cu", 37, 166, "/*"),                              # integrateRigidBody
    ("Kernels/rigidBodyKernels.cu", 262, 348, "GPUintegratorKernel"),            # GPUintegratorKernel
    ("Kernels/rigidBodyKernels.cu", 382, 421, "/*"),                             # computeGlobalAttributes
    ("Kernels/rigidBodyKernels.cu", 449, 456, "resetQuaternionKernel"),
    ("Kernels/RB_BVHKernels.cu", 13, 244, "maxOpF4"),                            # collideStaticSpheresBVH, collideBVHSoARigidBody
    ("Kernels/RB_BVHKernels.cu", 293, 442, "__global__"),                         # staticCollideBVHSoARigidBody
    ("Kernels/RB_BVHKernels.cu", 760, 876, "FindRigidBodyCollisionsBVHKernel"),
    ("Kernels/RB_BVHKernels.cu", 920, 1023, "FindAugmentedRealityCollisionsBVHKernel"),
    ("Kernels/RB_UniformGridKernels.cu", 112, 128, "calcGridPosAuxil"),          # grid pos / hash
    ("Kernels/RB_UniformGridKernels.cu", 419, 678, "__device__"),                # AR Baraff impulses: sphere pair, cell, kernel
    ("Kernels/RB_UniformGridKernels.cu", 730, 845, "__device__"),                # FindRigidBodyCollisionsUniformGrid cell + kernel
    ("Kernels/RB_UniformGridKernels.cu", 879, 1021, "__device__"),               # FindAugmentedRealityCollisionsUniformGrid cell + kernel
    ("WallCollisions.cu", 29, 35, "CreateIndexKernel"),
    ("WallCollisions.cu", 46, 129, "DetectWallCollisionKernel"),                 # + FindExactContactPoint, ComputeImpulseMagnitude
    ("WallCollisions.cu", 201, 276, "HandleWallCollisionKernelUnmapped"),
    ("Kernels/customRangeImageLoader.cu", 14, 113, "__global__ void RGBDloader("),
    ("Kernels/customRangeImageLoader.cu", 122, 177, "__global__ void computeNormals("),
]

# ParticleSystem member functions of the sequential-impulse path (host C++ with glm): the
# contact gather and the solver the reference's default update runs on the CPU, plus the
# contact-point helper they call.  They go to their own file, oracle/_ref/extracted_members.inc,
# which oracle/ref_cpu_driver.cpp includes after declaring a stand-in ParticleSystem class
# holding the members these bodies use.
MEMBER_RANGES = [
    ("Particles/CPU_Engine.cpp", 461, 473, "void ParticleSystem::findExactContactPoint("),
    ("Particles/updateFunctions.cpp", 1431, 1509, "void ParticleSystem::GatherRigidBodyCollisions()"),
    ("Particles/updateFunctions.cpp", 1511, 1578, "void ParticleSystem::GatherAugmentedRealityCollisions()"),
    ("Particles/updateFunctions.cpp", 1580, 1874, "void ParticleSystem::SequentialImpulseSolver()"),
]

# The part of ParticleSystem::initObject that turns a particle-body file into a body: centre of
# mass, per-model shift, the inertia sum (on a default-constructed glm::mat3, i.e. starting
# from the identity), glm::inverse and the hand-set tensors.  A block of statements, included
# into a function of oracle/ref_cpu_driver.cpp that supplies the locals it uses.
INIT_OBJECT_RANGE = [
    ("RigidBodies/RigidBodyAddition.cpp", 1576, 1756, "float maxDistance = -100000000;"),
]

STUB_HEADERS = {
    "cuda_gl_interop.h": "#pragma once\n",
    "helper_cuda_gl.h": "#pragma once\n",
    "curand.h": "#pragma once\n",
    "curand_kernel.h": "#pragma once\n",
}


def reference_root() -> Path:
    return Path(os.environ.get("AR_REFERENCE_ROOT", "/root/reference"))


def extract(ar_sim: Path, ranges=None) -> str:
    parts = []
    for rel, first, last, expect in (RANGES if ranges is None else ranges):
        lines = (ar_sim / rel).read_text(encoding="latin-1").splitlines()
        head = lines[first - 1]
        if expect not in head:
            raise RuntimeError(f"{rel}:{first} does not start with {expect!r} (found {head!r})")
        body = "\n".join(lines[first - 1:last])
        if body.count("{") != body.count("}"):
            raise RuntimeError(f"{rel}:{first}-{last} has unbalanced braces")
        parts.append(f'#line {first} "{ar_sim / rel}"\n{body}\n')
    return "\n".join(parts)


def build(verbose: bool = False) -> bool:
    root = reference_root()
    ar_sim = root / "AR_Sim"
    if not ar_sim.is_dir():
        if verbose:
            print(f"[ref_build] reference not found at {root}; skipping", file=sys.stderr)
        return False
    OUT.mkdir(exist_ok=True)
    shim = OUT / "shim"
    shim.mkdir(exist_ok=True)
    for name, text in STUB_HEADERS.items():
        (shim / name).write_text(text)
    (OUT / "extracted.inc").write_text(extract(ar_sim))
    (OUT / "extracted_members.inc").write_text(extract(ar_sim, MEMBER_RANGES))
    (OUT / "extracted_init_object.inc").write_text(extract(ar_sim, INIT_OBJECT_RANGE))
    so = OUT / "libref_cpu.so"
    cmd = [
        "g++", "-std=c++14", "-O2", "-fopenmp", "-fPIC", "-shared",
        "-ffp-contract=off", "-w",
        "-I", str(shim), "-I", str(OUT), "-I", str(HERE),
        "-I", "/usr/local/cuda/include",
        "-I", str(ar_sim / "BVHSource"), "-I", str(ar_sim / "Kernels"),
        "-I", str(ar_sim / "RigidBodies"),
        "-I", str(root / "Libs" / "common" / "inc"), "-I", str(root / "Libs" / "glm"),
        str(HERE / "ref_cpu_driver.cpp"), "-o", str(so),
    ]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return True


if __name__ == "__main__":
    ok = build(verbose=True)
    print("built" if ok else "skipped")
