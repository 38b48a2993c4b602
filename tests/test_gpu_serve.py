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
def test_native_server_results_equal_solo(ctx, broadphase):
    """The C++ request loop (ar_server_run): the same requests, results equal the scenes
    stepped alone bit for bit; a budget that holds only a few scenes at once makes requests
    queue behind resident ones; templates are shared by several requests (cloned on the
    device); a request of K = 0 returns its initial state."""
    rng = np.random.default_rng(9)
    pool = [scenes.small_scene(60 + i, nb_side=2 + i % 3, packed=(i % 2 == 1), r=1 / 128)
            for i in range(3)]
    reqs = []
    t = 0.0
    for i in range(12):
        t += float(rng.exponential(0.002)) if i >= 4 else 0.0
        k = 0 if i == 5 else int(rng.integers(3, 35))
        reqs.append(serve.Request(t, i, pool[i % 3], k))
    srv = serve.NativeServer(ctx, 64e9, tick_steps=4, broadphase=broadphase)
    stats = srv.run(reqs, keep_results=True)
    assert stats.completed == len(reqs) and stats.peak_resident >= 2
    # a budget of 2.5 of the largest scenes: resident bytes stay within it, and requests wait
    # for resident ones to leave
    d = api.make_desc(pool[2], api.broadphase_code(broadphase))
    from diploma_thesis_b200._lib import lib
    import ctypes as C
    budget = 2.5 * lib.ar_scene_footprint(C.byref(d))
    small = serve.NativeServer(ctx, budget, tick_steps=4, broadphase=broadphase)
    reqs2 = [serve.Request(0.0, 100 + i, r.scene, r.steps) for i, r in enumerate(reqs)]
    stats2 = small.run(reqs2, keep_results=True)
    assert stats2.completed == len(reqs2)
    assert stats2.peak_bytes <= budget and stats2.peak_resident < len(reqs2)
    srv.close()
    small.close()
    for r in reqs + reqs2:
        g = api.GpuScene(ctx, r.scene, broadphase=broadphase)
        if r.steps:
            g.step(r.steps, use_graph=False)
        alone = g.download()
        g.close()
        for k in ("pos", "quat", "vel", "angvel"):
            assert np.array_equal(alone[k], r.result[k]), (r.rid, k)
    ctx.check()


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
