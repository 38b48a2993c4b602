"""Re-sort from the previous step's order (csrc/ar_resort.cuh) against the radix sort from
scratch: a scene that has been stepped (its next step re-sorts) and a fresh scene given the same
state (its first step radix-sorts) must produce the same sorted keys and indices, the same
per-particle forces and the same body state, bit for bit -- with the ~1 % of particles that
change cell in a normal step, and with states under which nearly every particle does."""
import numpy as np
import pytest
import torch

from diploma_thesis_b200 import api, scenes

pytestmark = pytest.mark.gpu


def _sorted(gs: api.GpuScene):
    v = gs.step_view()
    n = v.num_particles
    keys = api.device_view(v.sorted_keys, n, torch.int32).cpu().numpy().view(np.uint32).copy()
    idx = api.device_view(v.sorted_idx, n, torch.int32).cpu().numpy().view(np.uint32).copy()
    pf = api.device_view(v.particle_force4, 4 * n, torch.float32).cpu().numpy().copy()
    return keys, idx, pf


def _compare_next_step(ctx, sc, warm_steps, perturb=None):
    """Step `a` warm_steps times, optionally replace its state, then step `a` (re-sort) and a
    fresh scene `b` holding the same state (radix sort) once each and compare."""
    a = api.GpuScene(ctx, sc)
    a.step(warm_steps, use_graph=True)
    state = a.download_state()
    if perturb is not None:
        state = np.ascontiguousarray(perturb(state))
        a.upload_state(state)
    b = api.GpuScene(ctx, sc)
    b.upload_state(state)
    a.step(1, use_graph=True)
    b.step(1, use_graph=True)
    ctx.check()
    ka, ia, fa = _sorted(a)
    kb, ib, fb = _sorted(b)
    assert np.all(ka[1:] >= ka[:-1])
    ties = ka[1:] == ka[:-1]
    assert np.all(ia[1:][ties] > ia[:-1][ties])
    assert np.array_equal(ka, kb) and np.array_equal(ia, ib)
    assert np.array_equal(fa, fb)
    assert np.array_equal(a.download_state(), b.download_state())
    a.close()
    b.close()
    return ka


@pytest.mark.parametrize("warm", [1, 7, 40])
def test_resort_equals_radix_sort_c0(ctx, warm):
    _compare_next_step(ctx, scenes.config0(0), warm)


def test_resort_equals_radix_sort_small_scenes(ctx):
    # fewer particles than one tile, and a few tiles with a partial last one
    for nb_side, packed in ((2, True), (5, False), (9, True)):
        _compare_next_step(ctx, scenes.small_scene(3, nb_side=nb_side, packed=packed,
                                                   r=1 / 128), 5)


def test_resort_equals_radix_sort_pile_2m(ctx):
    # the 2,097,152-particle pile: 1,024 tiles, 2^12 buckets over 25-bit keys
    _compare_next_step(ctx, scenes.config2(0), 12)


def _shift_x(cells):
    def f(state):
        s = state.copy()
        s[0, :, 0] += cells * (2.0 / 256.0)  # c0 cells are 2r = 2/256 wide
        return s
    return f


def _scatter_bodies(seed):
    def f(state):
        s = state.copy()
        rng = np.random.default_rng(seed)
        s[0, :, :3] = s[0, rng.permutation(s.shape[1]), :3]  # bodies swap places
        return s
    return f


@pytest.mark.parametrize("perturb", [_shift_x(1), _shift_x(37), _scatter_bodies(5)],
                         ids=["all_move_one_cell", "all_move_37_cells", "bodies_swapped"])
def test_resort_when_nearly_every_particle_moves(ctx, perturb):
    # an uploaded state far from the last step's: the re-sort meets movers in every tile and
    # buckets of more than 32 movers, and stays exact
    _compare_next_step(ctx, scenes.config0(0), 3, perturb)


def test_resort_in_batches_equals_solo(ctx):
    # several scenes: keys of each scene in its own cell range; the batch re-sorts after its
    # first step, the solo scenes too, and every result matches
    scs = [scenes.small_scene(s, nb_side=5, packed=True, r=1 / 128) for s in (11, 12, 13)]
    solo = [api.GpuScene(ctx, s) for s in scs]
    mem = [api.GpuScene(ctx, s) for s in scs]
    batch = api.Batch(ctx, mem)
    batch.step(30, use_graph=True)
    for g in solo:
        g.step(30, use_graph=True)
    ctx.check()
    for g, h in zip(solo, mem):
        assert np.array_equal(g.download_state(), h.download_state())
    batch.close()
    for g in solo + mem:
        g.close()


def _compare_next_step_bvh(ctx, sc, warm_steps, perturb=None):
    a = api.GpuScene(ctx, sc, broadphase="bvh")
    a.step(warm_steps, use_graph=True)
    state = a.download_state()
    if perturb is not None:
        state = np.ascontiguousarray(perturb(state))
        a.upload_state(state)
    b = api.GpuScene(ctx, sc, broadphase="bvh")
    b.upload_state(state)
    a.step(1, use_graph=True)
    b.step(1, use_graph=True)
    ctx.check()
    ka, ia, fa = _sorted(a)
    kb, ib, fb = _sorted(b)
    assert np.array_equal(ka, kb) and np.array_equal(ia, ib)
    assert np.array_equal(fa, fb)
    assert np.array_equal(a.download_state(), b.download_state())
    a.close()
    b.close()


@pytest.mark.parametrize("perturb", [None, _scatter_bodies(7)], ids=["steps", "bodies_swapped"])
def test_bvh_resort_equals_radix_sort(ctx, perturb):
    # the BVH step's 30-bit Morton keys (one scene) are re-sorted the same way
    _compare_next_step_bvh(ctx, scenes.config0(0), 9, perturb)


def test_bvh_resort_pile_2m(ctx):
    _compare_next_step_bvh(ctx, scenes.config2(0), 12)


def _shift_all(dx):
    def f(state):
        s = state.copy()
        s[0, :, 0] += dx
        return s
    return f


def test_resort_pile_2m_when_every_particle_moves(ctx):
    # the whole pile moved by five cells: every particle changes key, buckets hold up to ~2,000
    # movers (the ranking in global memory beyond 256 per bucket), and the result stays exact
    _compare_next_step(ctx, scenes.config2(0), 3, _shift_all(5.0 / 256.0))
