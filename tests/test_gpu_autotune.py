"""Autotuner candidates change speed, not contacts: every candidate (grid cell size, wrapped
grid size, block size, BVH) gives the same contact set and forces within 1e-5 relative; a
small bucket tunes end to end."""
import numpy as np
import pytest
import torch

from diploma_thesis_b200 import api, autotune, scenes

pytestmark = pytest.mark.gpu


def _forces(ctx, sc, kw):
    g = api.GpuScene(ctx, sc, **kw)
    g.step(1, use_graph=False)
    ctx.check()
    n = sc.num_particles
    f = api.device_view(g.step_view().particle_force4, 4 * n, torch.float32).cpu().numpy()
    g.close()
    return f.reshape(n, 4)[:, :3].copy()


def test_every_candidate_gives_the_same_contacts(ctx):
    sc = scenes.small_scene(11, nb_side=5, packed=True, r=1 / 128)
    ref = _forces(ctx, sc, {})
    touched = np.abs(ref).max(1) > 0
    assert touched.sum() > 100
    scale = np.maximum(np.abs(ref).max(1, keepdims=True), 1e-30)
    cands = [autotune.Choice(f, m, bs, 0.0) for f in autotune.CELL_FACTORS
             for m in autotune.GRID_MULTS for bs in (64, 256)]
    cands += [autotune.Choice(1.0, 0, bs, 0.0, "bvh") for bs in autotune.BLOCK_SIZES]
    for c in cands:
        f = _forces(ctx, sc, autotune.apply(sc, c))
        assert np.array_equal(np.abs(f).max(1) > 0, touched), c
        assert (np.abs(f - ref) / scale).max() <= 1e-5, c


def test_small_bucket_tunes(ctx, tmp_path):
    t = autotune.Tuner(ctx, tmp_path / "tune.json")
    c = t.choice(1000)
    assert c.ms_per_step > 0 and c.broadphase in ("grid", "bvh")
    assert (tmp_path / "tune.json").exists()
