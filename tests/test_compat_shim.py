"""include/arsim_compat.hpp against the reference's own wrapper declarations: a translation
unit that includes the reference headers (ParticleAuxiliaryFunctions.h, BVHcreation.h,
rigidBodyKernelWrappers.h) and the shim's definitions, takes the address of every wrapper
through the reference's declared type, and links against libarsim.so.  A signature that
differed would become an overload (ambiguous address) or an undefined symbol, and fail here.
Needs the reference checkout (read in place, nothing copied)."""
import os
import subprocess
import tempfile
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
REF = Path(os.environ.get("AR_REFERENCE_ROOT", "/root/reference"))
SHIM_STUBS = ROOT / "oracle" / "_ref" / "shim"

WRAPPERS = [
    # (name, reference declaration header)
    ("setParameters", "aux"), ("integrateSystem", "aux"), ("calcHash", "aux"),
    ("reorderDataAndFindCellStart", "aux"), ("collide", "aux"), ("sortParticles", "aux"),
    ("sortParticlesPreallocated", "aux"), ("createMortonCodesPreallocated", "aux"),
    ("initializeRadiiWrapper", "aux"), ("createMortonCodes", "bvh"),
    ("wrapperConstructRadixTreeSoA", "bvh"), ("wrapperConstructLeafNodesSoA", "bvh"),
    ("wrapperConstructInternalNodesSoA", "bvh"), ("integrateSystemRigidBodies", "rb"),
    ("GPUintegratorWrapper", "rb"), ("computeGlobalAttributesWrapper", "rb"),
    ("resetQuaternionWrapper", "rb"), ("ResetParticleImpulseWrapper", "rb"),
    ("FindAndHandleRigidBodyCollisionsUniformGridWrapper", "rb"),
    ("ReducePerParticleImpulses", "rb"), ("ReduceRigidBodyVariables", "rb"),
    ("WallCollisionWrapper", "rb"), ("collideBVHSoARigidBodyWrapper", "rb"),
    ("FindRigidBodyCollisionsBVHWrapper", "rb"),
]


@pytest.mark.skipif(not (REF / "AR_Sim").is_dir() or not SHIM_STUBS.is_dir(),
                    reason="needs the reference checkout and oracle/_ref stubs")
def test_shim_matches_reference_declarations_and_links():
    refs = "\n".join(f"  (void)static_cast<decltype(&{name})>(&{name});" for name, _ in WRAPPERS)
    src = f"""
#define GLM_FORCE_CUDA
#include <glm/glm.hpp>
#include <glm/gtc/quaternion.hpp>
#include "ParticleAuxiliaryFunctions.h"
#include "rigidBodyKernelWrappers.h"
#define ARSIM_COMPAT_IMPLEMENTATION
#include "arsim_compat.hpp"
int main() {{
{refs}
  return 0;
}}
"""
    a = REF / "AR_Sim"
    with tempfile.TemporaryDirectory() as td:
        cpp = Path(td) / "compat_check.cpp"
        cpp.write_text(src)
        exe = Path(td) / "compat_check"
        cmd = ["g++", "-std=c++14", "-w", "-I", str(SHIM_STUBS), "-I", "/usr/local/cuda/include",
               "-I", str(ROOT / "include"), "-I", str(a / "Kernels"), "-I", str(a / "BVHSource"),
               "-I", str(a / "RigidBodies"), "-I", str(a / "Particles"),
               "-I", str(REF / "Libs" / "common" / "inc"), "-I", str(REF / "Libs" / "glm"),
               str(cpp), "-o", str(exe), str(ROOT / "diploma_thesis_b200" / "libarsim.so"),
               "-L/usr/local/cuda/lib64", "-lcudart",
               f"-Wl,-rpath,{ROOT / 'diploma_thesis_b200'}"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-4000:]
