"""Failure paths, made on the host (no GPU fault): every device / pinned-host allocation of the
library goes through one wrapper that ar_test_fail_allocations can make fail.  Each case checks
the status code (AR_ERR_OOM, never a crash), that nothing half-built is handed out, and that
the same call succeeds, with results equal to the oracle's, once allocations work again."""
import ctypes as C

import numpy as np
import pytest
import torch

from diploma_thesis_b200 import _lib, api, scenes
from gpu_util import P, S, dev, empty, host
from oracle import cpu

pytestmark = pytest.mark.gpu

AR_ERR_OOM = 2


@pytest.fixture()
def inject():
    L = _lib.lib
    yield L.ar_test_fail_allocations
    L.ar_test_fail_allocations(-1)


def test_context_creation_out_of_memory(inject):
    L = _lib.lib
    for after in (0, 1):  # the error word, then its pinned host mirror
        inject(after)
        h = C.c_void_p()
        assert L.ar_ctx_create(0, C.byref(h)) == AR_ERR_OOM
        assert not h.value
        assert b"allocation failed" in L.ar_last_error()
    inject(-1)
    h = C.c_void_p()
    assert L.ar_ctx_create(0, C.byref(h)) == 0 and h.value
    assert L.ar_ctx_destroy(h) == 0


def test_scene_and_step_out_of_memory_then_recover(ctx, inject):
    L = _lib.lib
    sc = scenes.small_scene(3, nb_side=4, packed=True, r=1 / 128)
    inject(0)
    with pytest.raises(_lib.ArError) as e:
        api.GpuScene(ctx, sc)
    assert e.value.status == AR_ERR_OOM
    inject(-1)
    gs = api.GpuScene(ctx, sc)
    # the first step builds the scene's batch workspace: fail each of its first allocations
    for after in (0, 1, 3, 7):
        inject(after)
        assert L.ar_step(ctx.handle, gs.handle, 1, 1, S()) == AR_ERR_OOM
        inject(-1)
    gs.step(4, use_graph=True)
    ctx.check()
    ref = cpu.step(sc, 4)
    got = gs.download()
    for k in ("pos", "quat", "vel", "angvel"):
        assert np.array_equal(got[k], ref[k]), k
    gs.close()


def test_bvh_workspace_out_of_memory_then_recover(ctx, inject):
    L = _lib.lib
    sc = scenes.small_scene(4, nb_side=4, packed=True, r=1 / 128)
    gs = api.GpuScene(ctx, sc, broadphase="bvh")
    inject(14)  # past the grid workspace (14 arrays), into the BVH arrays
    assert L.ar_step(ctx.handle, gs.handle, 1, 0, S()) == AR_ERR_OOM
    inject(-1)
    gs.step(3, use_graph=False)
    ctx.check()
    ref = cpu.step(sc, 3, broadphase="bvh")
    got = gs.download()
    for k in ("pos", "quat", "vel", "angvel"):
        assert np.array_equal(got[k], ref[k]), k
    gs.close()


def test_scratch_arena_out_of_memory(inject):
    L = _lib.lib
    h = C.c_void_p()
    assert L.ar_ctx_create(0, C.byref(h)) == 0
    n = 100_000
    keys = dev(np.arange(n, dtype=np.uint32)[::-1].copy())
    ko, vo = empty(n, torch.int32), empty(n, torch.int32)
    inject(0)
    assert L.ar_radix_sort_pairs_u32(h, P(keys), None, P(ko), P(vo), n, 0, 17, S()) == AR_ERR_OOM
    inject(-1)
    assert L.ar_radix_sort_pairs_u32(h, P(keys), None, P(ko), P(vo), n, 0, 17, S()) == 0
    assert np.array_equal(host(vo, np.uint32), np.arange(n, dtype=np.uint32)[::-1])
    assert L.ar_ctx_status(h, S()) == 0
    assert L.ar_ctx_destroy(h) == 0
