"""The reference's own GPU step (oracle/_ref/libref_gpu.so, built from the reference's CUDA
sources), checked against the reference's CPU build on the same scene, so that the timings
oracle/ref_gpu_bench.py reports for it are timings of the reference's real step.

Both run REFERENCE semantics from the same state for three steps on a packed scene with
contacts.  The GPU build sorts with CUB and sums the per-body impulses as prefix-sum
differences of CUB scans; the CPU build uses a stable sort (the same permutation) and
sequential scans, so the sums agree to rounding: velocities within 1e-5 absolute + 1e-3
relative, positions within 1e-6 absolute."""
import numpy as np
import pytest

from diploma_thesis_b200 import scenes
from oracle import cpu, ref, ref_gpu
from oracle.ref_step import ReferenceCPUStep

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not (ref_gpu.available() and ref.available()),
                    reason="the reference GPU / CPU builds are not present")
def test_reference_gpu_step_matches_reference_cpu_step(ctx):
    sc = scenes.small_scene(8, nb_side=4, packed=True, r=1 / 128)
    grid = cpu.scene_grid(sc)
    gpu = ref_gpu.RefGpuStep(sc, grid)
    host = ReferenceCPUStep(sc, grid)
    try:
        for _ in range(3):
            ms, wall = gpu.step()
            host.step()
            assert np.all(np.isfinite(ms)) and np.all(ms >= 0) and wall > 0
        pos, vel = gpu.bodies()
    finally:
        gpu.close()
    assert np.allclose(vel[:, :3], host.st["vel"][:, :3], rtol=1e-3, atol=1e-5)
    assert np.allclose(pos[:, :3], host.st["cms"][:, :3], rtol=0, atol=1e-6)
    # the step moved the bodies (contacts and gravity acted)
    assert not np.array_equal(vel[:, :3], sc.body_vel[:, :3])
