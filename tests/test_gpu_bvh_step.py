"""The fused step with the BVH broad phase (Morton keys -> onesweep sort of 32-bit keys, or
64-bit keys for more than 4 scenes -> Karras tree -> refit -> stackless walk) against the oracle's float32 restatement (bit-exact), batched
against solo, and against the grid broad phase (same contacts, forces within 1e-5 relative)."""
import numpy as np
import pytest
import torch

from diploma_thesis_b200 import api, scenes
from diploma_thesis_b200._lib import ArError
from oracle import cpu

pytestmark = pytest.mark.gpu


def _keys(v) -> np.ndarray:
    """Sorted BVH keys as uint64 (32-bit keys when they fit, at most 4 scenes)."""
    n = v.num_particles
    assert v.key_bytes == (4 if v.key_bits <= 32 else 8)
    if v.key_bytes == 4:
        k = api.device_view(v.sorted_keys, n, torch.int32).cpu().numpy().view(np.uint32)
        return k.astype(np.uint64)
    return api.device_view(v.sorted_keys, 2 * n, torch.int32).cpu().numpy().view(np.uint64)


def _view(gs: api.GpuScene):
    v = gs.step_view()
    n = v.num_particles
    assert v.broadphase == 1 and not v.cells2
    keys = _keys(v)
    idx = api.device_view(v.sorted_idx, n, torch.int32).cpu().numpy().view(np.uint32)
    pf = api.device_view(v.particle_force4, 4 * n, torch.float32).cpu().numpy().reshape(n, 4)
    return keys, idx, pf


@pytest.mark.parametrize("seed,packed", [(1, True), (2, False), (6, True)])
def test_bvh_one_step_bit_exact_with_oracle(ctx, seed, packed):
    sc = scenes.small_scene(seed, nb_side=5, packed=packed, r=1 / 128)
    gs = api.GpuScene(ctx, sc, broadphase="bvh")
    gs.step(1, use_graph=False)
    ctx.check()
    ref = cpu.step(sc, 1, broadphase="bvh")
    keys, idx, pf = _view(gs)
    assert np.array_equal(keys, ref["skeys"]) and np.array_equal(idx, ref["sidx"])
    assert np.array_equal(pf, ref["pforce"])
    if packed:
        assert (np.abs(pf).sum(1) > 0).sum() > 100
    got = gs.download()
    for k in ("pos", "quat", "vel", "angvel"):
        assert np.array_equal(got[k], ref[k]), k
    gs.close()


def test_bvh_tree_matches_oracle_radix_tree(ctx):
    sc = scenes.small_scene(4, nb_side=4, packed=True, r=1 / 128)
    gs = api.GpuScene(ctx, sc, broadphase="bvh")
    gs.step(1, use_graph=False)
    ctx.check()
    v = gs.step_view()
    n = v.num_particles
    keys = _keys(v)
    left = api.device_view(v.tree_left, 2 * n, torch.int32).cpu().numpy()
    right = api.device_view(v.tree_right, 2 * n, torch.int32).cpu().numpy()
    parent = api.device_view(v.tree_parent, 2 * n, torch.int32).cpu().numpy()
    t = cpu.radix_tree(keys.copy())
    assert np.array_equal(left[n:2 * n - 1], t["left"][n:2 * n - 1])
    assert np.array_equal(right[n:2 * n - 1], t["right"][n:2 * n - 1])
    assert np.array_equal(parent[:n], t["parent"][:n])
    assert parent[n] == -1
    gs.close()


def test_bvh_hundred_steps_bit_exact_graph_and_eager(ctx):
    sc = scenes.small_scene(3, nb_side=4, packed=True, r=1 / 128)
    a = api.GpuScene(ctx, sc, broadphase="bvh")
    b = api.GpuScene(ctx, sc, broadphase="bvh")
    a.step(100, use_graph=True)
    b.step(100, use_graph=False)
    ctx.check()
    ga, gb = a.download(), b.download()
    ref = cpu.step(sc, 100, broadphase="bvh")
    for k in ("pos", "quat", "vel", "angvel"):
        assert np.array_equal(ga[k], ref[k]), k
        assert np.array_equal(gb[k], ref[k]), k
    f64 = cpu.step_f64(sc, 100)
    assert np.abs(ga["pos"][:, :3] - f64["pos"][:, :3]).max() <= 1e-3 * sc.radius
    a.close()
    b.close()


@pytest.mark.parametrize("sides", [(3, 5, 2, 4, 1, 4), (3, 2, 4)])  # 64- and 32-bit keys
def test_bvh_batch_equals_solo_bit_for_bit(ctx, sides):
    group = []
    for i, side in enumerate(sides):
        sc = scenes.small_scene(i + 20, nb_side=side, packed=(i % 2 == 0), r=1 / 128)
        group.append(sc)
    solo = [api.GpuScene(ctx, sc, broadphase="bvh") for sc in group]
    batched = [api.GpuScene(ctx, sc, broadphase="bvh") for sc in group]
    for s in solo:
        s.step(7, use_graph=False)
    batch = api.Batch(ctx)
    batch.set_scenes(batched)
    batch.step(7, use_graph=True)
    ctx.check()
    for s, b in zip(solo, batched):
        x, y = s.download(), b.download()
        for k in ("pos", "quat", "vel", "angvel"):
            assert np.array_equal(x[k], y[k]), k
    batch.close()
    for s in solo + batched:
        s.close()


def test_bvh_forces_match_grid_forces(ctx):
    sc = scenes.small_scene(7, nb_side=5, packed=True, r=1 / 128)
    g = api.GpuScene(ctx, sc)
    b = api.GpuScene(ctx, sc, broadphase="bvh")
    g.step(1, use_graph=False)
    b.step(1, use_graph=False)
    ctx.check()
    n = sc.num_particles
    fg = api.device_view(g.step_view().particle_force4, 4 * n, torch.float32).cpu().numpy()
    fb = api.device_view(b.step_view().particle_force4, 4 * n, torch.float32).cpu().numpy()
    fg, fb = fg.reshape(n, 4)[:, :3], fb.reshape(n, 4)[:, :3]
    touched = np.abs(fg).max(1) > 0
    assert touched.sum() > 100
    assert np.array_equal(touched, np.abs(fb).max(1) > 0)
    scale = np.maximum(np.abs(fg).max(1, keepdims=True), 1e-30)
    assert (np.abs(fg - fb) / scale).max() <= 1e-5
    g.close()
    b.close()


def test_mixed_broadphase_batch_is_rejected(ctx):
    a = api.GpuScene(ctx, scenes.small_scene(1, nb_side=2), broadphase="grid")
    b = api.GpuScene(ctx, scenes.small_scene(2, nb_side=2), broadphase="bvh")
    batch = api.Batch(ctx)
    with pytest.raises(ArError):
        batch.set_scenes([a, b])
    batch.close()
    a.close()
    b.close()


def test_batch_reconfigured_across_broadphases(ctx):
    """One batch object re-targeted grid -> BVH -> BVH subset -> grid after graph steps: each
    layout's results equal the same scenes stepped alone."""
    scs = [scenes.small_scene(60 + i, nb_side=2 + i % 2, packed=True, r=1 / 128)
           for i in range(3)]
    batch = api.Batch(ctx)
    for bp, idx in (("grid", [0, 1, 2]), ("bvh", [0, 1, 2]), ("bvh", [2, 0]), ("grid", [1])):
        members = [api.GpuScene(ctx, scs[i], broadphase=bp) for i in idx]
        alone = [api.GpuScene(ctx, scs[i], broadphase=bp) for i in idx]
        batch.set_scenes(members)
        batch.step(4, use_graph=True)
        for a in alone:
            a.step(4, use_graph=True)
        ctx.check()
        for m, a in zip(members, alone):
            x, y = m.download(), a.download()
            for k in ("pos", "quat", "vel", "angvel"):
                assert np.array_equal(x[k], y[k]), (bp, k)
        for g in members + alone:
            g.close()
    batch.close()
