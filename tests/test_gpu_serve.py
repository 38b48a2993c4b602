"""Continuous batching on the device: every served request's result equals the same scene
stepped alone for K steps, bit for bit, whatever scenes shared its batches; step budgets
freeze scenes after exactly K steps; scene memory is released in stream order and reused."""
import numpy as np
import pytest

from diploma_thesis_b200 import api, scenes, serve

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("broadphase", ["grid", "bvh"])
def test_served_results_equal_solo(ctx, broadphase):
    rng = np.random.default_rng(5)
    pool = [scenes.small_scene(40 + i, nb_side=2 + i % 3, packed=(i % 2 == 0), r=1 / 128)
            for i in range(4)]
    reqs = []
    t = 0.0
    for i in range(10):
        t += float(rng.exponential(0.003)) if i >= 3 else 0.0  # three at once, then Poisson
        reqs.append(serve.Request(t, i, pool[i % 4], int(rng.integers(3, 40))))
    srv = serve.Server(ctx, 64e9, tick_steps=5, keep_results=True, broadphase=broadphase)
    stats = srv.run(reqs)
    srv.close()
    assert stats.completed == len(reqs)
    assert stats.peak_resident >= 2  # requests overlapped on the device
    for r in reqs:
        g = api.GpuScene(ctx, r.scene, broadphase=broadphase)
        g.step(r.steps, use_graph=False)
        alone = g.download()
        g.close()
        for k in ("pos", "quat", "vel", "angvel"):
            assert np.array_equal(alone[k], r.result[k]), (r.rid, k)


@pytest.mark.parametrize("broadphase", ["grid", "bvh"])
def test_step_budgets_freeze_scenes_after_k_steps(ctx, broadphase):
    scs = [scenes.small_scene(70 + i, nb_side=3, packed=True, r=1 / 128) for i in range(3)]
    budgets = [4, -1, 9]
    members = [api.GpuScene(ctx, sc, broadphase=broadphase) for sc in scs]
    batch = api.Batch(ctx)
    batch.set_scenes(members, budgets)
    batch.step(5, use_graph=True)
    batch.step(7, use_graph=False)  # 12 steps in all
    ctx.check()
    for sc, m, k in zip(scs, members, budgets):
        alone = api.GpuScene(ctx, sc, broadphase=broadphase)
        alone.step(12 if k < 0 else k, use_graph=False)
        x, y = m.download(), alone.download()
        for key in ("pos", "quat", "vel", "angvel"):
            assert np.array_equal(x[key], y[key]), (k, key)
        alone.close()
    batch.close()
    for m in members:
        m.close()


def test_stream_ordered_destroy_and_reuse(ctx):
    import torch
    st = torch.cuda.Stream()
    sc = scenes.small_scene(80, nb_side=3, packed=True, r=1 / 128)
    ref = api.GpuScene(ctx, sc)
    ref.step(6, use_graph=False)
    want = ref.download()
    ref.close()
    for _ in range(4):  # freed blocks go back to the pool and are handed out again
        a = api.GpuScene(ctx, sc, stream=st)
        b = api.Batch(ctx, [a])
        b.step(6, use_graph=True, stream=st)
        host = a.download_async(st)
        b.set_scenes([])
        a.close_async(st)
        st.synchronize()
        for key in ("pos", "quat", "vel", "angvel"):
            assert np.array_equal(host[key], want[key]), key
        b.close()
    ctx.check()
