"""Parity at the benchmarked sizes: the fused step on the 2,097,152-particle pile (the bench's
default workload) and on a 531,441-particle packed scene, with both broad phases, against the
oracle's float32 restatement, bit for bit; and the 4,096-cube plain scene over 100 steps.

These sizes take the paths that small scenes never reach:
  * the grid step's cell-key sort at n >= 2^19 runs its 8-bit digit passes on 512-thread tiles
    ranked by warp match.any (onesweep_kernel<u32, 512, 8, true>) and, for the pile's 25-bit
    keys (256 x 512 x 256 wrapped grid), a 9-bit pass on 512-thread tiles ranked by ballots;
  * the BVH step sorts 30-bit Morton keys on 512-thread tiles in four passes (8, 8, 8, 6);
  * the cell table holds 2^25 (pile) or 2^23 (packed) entries, far beyond L2.

Each case compares the last step's sorted keys, the permutation (sorted particle indices), the
per-particle forces and the body state (position, orientation, velocity, angular velocity)
with the oracle.  The pile is checked twice: over its first steps, and over two steps started
from its state after 1,500 GPU steps, when bodies drifting inside their layers have come into
contact (the oracle takes that state as its input, so both sides advance the same state)."""
import numpy as np
import pytest
import torch

from diploma_thesis_b200 import api, scenes
from oracle import cpu

pytestmark = pytest.mark.gpu

STATE_KEYS = ("pos", "quat", "vel", "angvel")


@pytest.fixture(scope="module")
def pile():
    return scenes.config2(0)


@pytest.fixture(scope="module")
def packed():
    # 27^3 cubes of 27 particles, neighbours in contact from the first step
    return scenes.small_scene(7, nb_side=27, k=3, packed=True, r=1 / 512)


def _last_step(gs: api.GpuScene, bvh: bool):
    v = gs.step_view()
    n = v.num_particles
    if bvh and v.key_bytes == 8:
        keys = api.device_view(v.sorted_keys, 2 * n, torch.int32).cpu().numpy().view(np.uint64)
    else:
        keys = api.device_view(v.sorted_keys, n, torch.int32).cpu().numpy().view(np.uint32)
    idx = api.device_view(v.sorted_idx, n, torch.int32).cpu().numpy().view(np.uint32)
    pf = api.device_view(v.particle_force4, 4 * n, torch.float32).cpu().numpy().reshape(n, 4)
    return keys, idx, pf, v


def _compare(gs, ref, bvh):
    keys, idx, pf, v = _last_step(gs, bvh)
    ref_keys = ref["skeys"]
    if bvh:
        keys = keys.astype(np.uint64)
    assert np.array_equal(keys, ref_keys), "sorted keys differ"
    assert np.array_equal(idx, ref["sidx"]), "sort permutation differs"
    assert np.array_equal(pf, ref["pforce"]), "per-particle forces differ"
    got = gs.download()
    for k in STATE_KEYS:
        assert np.array_equal(got[k], ref[k]), k
    return pf, v


@pytest.mark.parametrize("broadphase", ["grid", "bvh"])
def test_pile_first_steps_bit_exact(ctx, pile, broadphase):
    bvh = broadphase == "bvh"
    gs = api.GpuScene(ctx, pile, broadphase=broadphase)
    assert gs.num_particles == 2_097_152 and gs.num_particles >= 1 << 19
    if not bvh:
        assert gs.grid_info()[2] == [256, 512, 256]
    gs.step(3, use_graph=True)
    ctx.check()
    _, v = _compare(gs, cpu.step(pile, 3, broadphase=broadphase), bvh)
    assert v.key_bits == (25 if not bvh else 30)
    gs.close()


@pytest.mark.parametrize("broadphase", ["grid", "bvh"])
def test_pile_mid_trajectory_bit_exact(ctx, pile, broadphase):
    bvh = broadphase == "bvh"
    gs = api.GpuScene(ctx, pile, broadphase=broadphase)
    gs.step(1500, use_graph=True)
    ctx.check()
    state = gs.download()
    assert all(np.isfinite(state[k]).all() for k in STATE_KEYS)
    gs.step(2, use_graph=True)
    ctx.check()
    ref = cpu.step(pile, 2, state=state, broadphase=broadphase)
    pf, _ = _compare(gs, ref, bvh)
    # particle-particle contacts are present (wall contacts aside: the pile has not reached
    # the floor yet, and the side walls are 3 cells from the outermost bodies at most)
    assert (np.abs(pf[:, :3]).sum(1) > 0).sum() > 1000
    gs.close()


@pytest.mark.parametrize("broadphase", ["grid", "bvh"])
def test_packed_half_million_bit_exact(ctx, packed, broadphase):
    bvh = broadphase == "bvh"
    gs = api.GpuScene(ctx, packed, broadphase=broadphase)
    assert gs.num_particles == 531_441 and gs.num_particles >= 1 << 19
    gs.step(2, use_graph=False)
    ctx.check()
    pf, _ = _compare(gs, cpu.step(packed, 2, broadphase=broadphase), bvh)
    assert (np.abs(pf[:, :3]).sum(1) > 0).sum() > 400_000
    gs.close()


def test_config0_hundred_steps_bit_exact_and_near_fp64(ctx):
    sc = scenes.config0(0)
    gs = api.GpuScene(ctx, sc)
    gs.step(100, use_graph=True)
    ctx.check()
    got = gs.download()
    ref = cpu.step(sc, 100)
    for k in STATE_KEYS:
        assert np.array_equal(got[k], ref[k]), k
    f64 = cpu.step_f64(sc, 100)
    # stated trajectory tolerance: body positions within 1e-3 r of FP64 after 100 steps
    # (float32 rounding of x += dt v over 100 steps at |x| ~ 0.5 is ~3e-6 = 0.8e-3 r)
    assert np.abs(got["pos"][:, :3] - f64["pos"][:, :3]).max() <= 1e-3 * sc.radius
    gs.close()
