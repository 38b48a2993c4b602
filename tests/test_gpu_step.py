"""The fused step (ar_step / ar_batch_step) against the oracle's float32 restatement
(bit-exact), against the FP64 oracle (stated tolerances), and batched against solo."""
import ctypes as C

import numpy as np
import pytest
import torch

from diploma_thesis_b200 import api, scenes
from gpu_util import host
from oracle import cpu

pytestmark = pytest.mark.gpu


def _scene_state(gs: api.GpuScene) -> dict:
    return gs.download()


def _sorted_arrays(gs: api.GpuScene):
    v = gs.step_view()
    n = v.num_particles
    keys = api.device_view(v.sorted_keys, n, torch.int32).cpu().numpy().view(np.uint32)
    idx = api.device_view(v.sorted_idx, n, torch.int32).cpu().numpy().view(np.uint32)
    pf = api.device_view(v.particle_force4, 4 * n, torch.float32).cpu().numpy().reshape(n, 4)
    return keys, idx, pf


@pytest.mark.parametrize("seed,packed", [(1, True), (2, False)])
def test_one_step_bit_exact_with_oracle(ctx, seed, packed):
    sc = scenes.small_scene(seed, nb_side=5, packed=packed, r=1 / 128)
    gs = api.GpuScene(ctx, sc)
    o, c, d = gs.grid_info()
    assert (o, d) == (cpu.scene_grid(sc)[0], cpu.scene_grid(sc)[2])
    gs.step(1, use_graph=False)
    ctx.check()
    ref = cpu.step(sc, 1)
    got = gs.download()
    keys, idx, pf = _sorted_arrays(gs)
    assert np.array_equal(keys, ref["skeys"]) and np.array_equal(idx, ref["sidx"])
    assert np.array_equal(pf, ref["pforce"])
    if packed:
        assert (np.abs(pf).sum(1) > 0).sum() > 100
    for k in ("pos", "quat", "vel", "angvel"):
        assert np.array_equal(got[k], ref[k]), k
    gs.close()


def test_hundred_steps_bit_exact_and_near_fp64(ctx):
    sc = scenes.small_scene(3, nb_side=4, packed=True, r=1 / 128)
    gs = api.GpuScene(ctx, sc)
    gs.step(100, use_graph=True)
    ctx.check()
    got = gs.download()
    ref = cpu.step(sc, 100)
    for k in ("pos", "quat", "vel", "angvel"):
        assert np.array_equal(got[k], ref[k]), k
    f64 = cpu.step_f64(sc, 100)
    # trajectory tolerance against FP64 after 100 steps: 1e-3 r in position
    assert np.abs(got["pos"][:, :3] - f64["pos"][:, :3]).max() <= 1e-3 * sc.radius
    gs.close()


def test_graph_and_eager_agree(ctx):
    sc = scenes.small_scene(5, nb_side=4, packed=True, r=1 / 128)
    a, b = api.GpuScene(ctx, sc), api.GpuScene(ctx, sc)
    a.step(17, use_graph=True)
    b.step(17, use_graph=False)
    da, db = a.download(), b.download()
    for k in da:
        assert np.array_equal(da[k], db[k]), k
    a.close()
    b.close()


def test_batch_equals_solo_bit_for_bit(ctx):
    sizes = [(2, 3), (3, 4), (4, 3), (5, 5)]
    solo, members = [], []
    for i, (seed, side) in enumerate(sizes):
        sc = scenes.small_scene(seed + 10, nb_side=side, packed=(i % 2 == 0), r=1 / 128,
                                box=0.6 + 0.2 * i)
        solo.append(api.GpuScene(ctx, sc))
        members.append(api.GpuScene(ctx, sc))
    batch = api.Batch(ctx, members)
    batch.step(25)
    for s in solo:
        s.step(25)
    ctx.check()
    for s, m in zip(solo, members):
        a, b = s.download(), m.download()
        for k in a:
            assert np.array_equal(a[k], b[k]), k
    # change membership mid-run: remaining scenes continue identically
    batch.set_scenes(members[1:3])
    batch.step(10)
    for s in solo[1:3]:
        s.step(10)
    for s, m in zip(solo[1:3], members[1:3]):
        a, b = s.download(), m.download()
        for k in a:
            assert np.array_equal(a[k], b[k]), k
    batch.close()
    for s in solo + members:
        s.close()


def test_nan_state_is_reported(ctx):
    sc = scenes.small_scene(8, nb_side=2, r=1 / 128)
    sc.body_vel[1, 0] = np.nan
    gs = api.GpuScene(ctx, sc)
    gs.step(1, use_graph=False)
    assert ctx.status() == 4  # AR_ERR_NAN
    assert ctx.status() == 0
    gs.close()


def test_invalid_scene_arguments(ctx):
    from diploma_thesis_b200 import _lib
    sc = scenes.small_scene(1, nb_side=2)
    d = api.make_desc(sc)
    d.block_size = 100
    init = _lib.SceneInit()
    h = C.c_void_p()
    assert _lib.lib.ar_scene_create(ctx.handle, C.byref(d), C.byref(init), None, C.byref(h)) == 1
    with pytest.raises(_lib.ArError):
        sc2 = scenes.small_scene(1, nb_side=2)
        sc2.body_offsets = sc2.body_offsets.copy()
        sc2.body_offsets[-1] += 1
        api.GpuScene(ctx, sc2)


def test_config0_first_steps_bit_exact(ctx):
    sc = scenes.config0(0)
    gs = api.GpuScene(ctx, sc)
    assert gs.grid_info()[2] == [128, 128, 128]
    gs.step(2, use_graph=True)
    ctx.check()
    ref = cpu.step(sc, 2)
    got = gs.download()
    for k in ("pos", "quat", "vel", "angvel"):
        assert np.array_equal(got[k], ref[k]), k
    gs.close()


def test_model_matrices_for_the_renderer(ctx):
    sc = scenes.small_scene(12, nb_side=3, packed=True, r=1 / 128)
    gs = api.GpuScene(ctx, sc)
    gs.step(5, use_graph=True)
    m = gs.model_matrices().cpu().numpy()
    st = gs.download()
    R = scenes.quat_to_matrix(st["quat"].astype(np.float64))
    # glm column-major: m[b, c, r] = element (r, c); column 3 holds the centre
    assert np.allclose(m[:, :3, :3], np.transpose(R, (0, 2, 1)), atol=2e-6)
    assert np.array_equal(m[:, 3, :3], st["pos"][:, :3])
    assert np.all(m[:, :3, 3] == 0) and np.all(m[:, 3, 3] == 1)
    gs.close()


def _cell_table(gs: api.GpuScene):
    v = gs.step_view()
    cells = api.device_view(v.cells2, 2 * v.num_cells, torch.int32).cpu().numpy().view(np.uint32)
    return cells.reshape(-1, 2)


def test_cell_epochs_recur_without_stale_entries(ctx):
    """Epochs repeat every 255 steps; the rolling slice clear keeps stale entries from
    matching, so 600 graph-replayed steps stay bit-exact."""
    sc = scenes.small_scene(4, nb_side=4, packed=True, r=1 / 128)
    gs = api.GpuScene(ctx, sc)
    gs.step(600, use_graph=True)
    ctx.check()
    got = gs.download()
    ref = cpu.step(sc, 600)
    for k in ("pos", "quat", "vel", "angvel"):
        assert np.array_equal(got[k], ref[k]), k
    gs.close()


def test_cell_table_entries(ctx):
    """Every occupied cell: first sorted slot, saturating count, this step's epoch and the body
    tag; a 4^3 wrapped grid crowds more than 31 particles into some cells, whose end is then
    found from the sorted keys (results stay bit-exact)."""
    sc = scenes.small_scene(6, nb_side=5, packed=True, r=1 / 128)
    sc.grid_log2 = (2, 2, 2)
    gs = api.GpuScene(ctx, sc)
    steps = 3
    gs.step(steps, use_graph=False)
    ctx.check()
    ref = cpu.step(sc, steps)
    got = gs.download()
    for k in ("pos", "quat", "vel", "angvel"):
        assert np.array_equal(got[k], ref[k]), k
    keys, idx, pf = _sorted_arrays(gs)
    assert np.array_equal(pf, ref["pforce"])
    table = _cell_table(gs)
    body = sc.body_index()
    uk, first, cnt = np.unique(keys, return_index=True, return_counts=True)
    assert cnt.max() > 31
    meta = table[uk, 1]
    assert np.array_equal(table[uk, 0], first)
    assert np.array_equal(meta & 31, np.minimum(cnt, 31))
    assert np.all(((meta >> 5) & 255) == steps % 255 + 1)
    sb = body[idx]
    single = np.minimum.reduceat(sb, first) == np.maximum.reduceat(sb, first)
    assert np.array_equal(meta >> 13, np.where(single, sb[first] + 1, 0))
    gs.close()


def test_packed_state_transfers(ctx):
    """ar_scene_upload_state / ar_scene_download_state move the same bytes as the four-array
    calls, with one copy each way (the device arrays sit at a padded pitch)."""
    sc = scenes.small_scene(9, nb_side=3, packed=True, r=1 / 128)  # 27 bodies: padded pitch
    a, b = api.GpuScene(ctx, sc), api.GpuScene(ctx, sc)
    a.step(5, use_graph=False)
    got = a.download()
    packed = a.download_state()
    assert np.array_equal(packed, np.stack([got[k] for k in ("pos", "quat", "vel", "angvel")]))
    pinned = torch.empty((4, sc.num_bodies, 4), dtype=torch.float32).pin_memory().numpy()
    a.download_state(pinned, wait=False)
    torch.cuda.synchronize()
    assert np.array_equal(pinned, packed)
    # b takes a's state through the packed upload; both then step identically
    b.upload_state(packed)
    a.step(3, use_graph=False)
    b.step(3, use_graph=False)
    ctx.check()
    x, y = a.download(), b.download()
    for k in x:
        assert np.array_equal(x[k], y[k]), k
    a.close()
    b.close()


def test_step_io_round_trip(ctx):
    """ar_scene_step_io (upload, n graph steps, download in one call) gives what the three
    separate calls give, into the same pinned array it read from."""
    sc = scenes.small_scene(13, nb_side=3, packed=True, r=1 / 128)
    a, b = api.GpuScene(ctx, sc), api.GpuScene(ctx, sc)
    a.step(4, use_graph=False)
    state = a.download_state()
    pinned = torch.empty((4, sc.num_bodies, 4), dtype=torch.float32).pin_memory().numpy()
    pinned[:] = state
    for _ in range(3):
        b.step_io(pinned, 2, pinned)      # b: state in, 2 steps, state back, six steps in all
        a.step(2, use_graph=True)
    got = a.download_state()
    assert np.array_equal(pinned, got)
    a.close()
    b.close()

