"""Continuous batching on the device: every served request's result equals the same scene
stepped alone for K steps, bit for bit, whatever scenes shared its batches."""
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
