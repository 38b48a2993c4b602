"""A static point cloud attached to a scene (ar_scene_set_static_cloud): the fused step with
the simulateAR branch of updateUniformGridDEM (RigidBodies/UniformGridUpdate.cpp:967-969)
against the oracle's float32 restatement (bit-exact), detached, batched against solo, and fed
from a depth image through ar_range_image_cloud / ar_range_image_normals."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import golden
from diploma_thesis_b200 import api, scenes
from diploma_thesis_b200._lib import ArError, call
from oracle import cpu

pytestmark = pytest.mark.gpu

STATE = ("pos", "quat", "vel", "angvel")


def random_cloud(seed: int, m: int, lo: float, hi: float):
    """m points uniform in [lo, hi]^3 with random unit normals (float32)."""
    rng = np.random.default_rng(seed)
    pos = np.zeros((m, 4), np.float32)
    pos[:, :3] = rng.uniform(lo, hi, (m, 3))
    n = rng.normal(size=(m, 3))
    nrm = np.zeros((m, 4), np.float32)
    nrm[:, :3] = n / np.linalg.norm(n, axis=1, keepdims=True)
    return pos, nrm


def _dev(a: np.ndarray) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _forces(gs: api.GpuScene) -> np.ndarray:
    v = gs.step_view()
    n = v.num_particles
    return api.device_view(v.particle_force4, 4 * n, torch.float32).cpu().numpy().reshape(n, 4)


def test_cloud_step_bit_exact_with_oracle(ctx):
    sc = scenes.small_scene(5, nb_side=4, r=1 / 128)
    cloud = random_cloud(11, 20000, 0.2, 0.8)
    gs = api.GpuScene(ctx, sc)
    gs.set_static_cloud(_dev(cloud[0]), _dev(cloud[1]))
    gs.step(1, use_graph=False)
    ctx.check()
    ref = cpu.step(sc, 1, cloud=cloud)
    plain = cpu.step(sc, 1)
    pf = _forces(gs)
    assert np.array_equal(pf, ref["pforce"])
    changed = (ref["pforce"][:, :3] != plain["pforce"][:, :3]).any(1).sum()
    assert changed > 100, changed  # the cloud pushes many particles
    got = gs.download()
    for k in STATE:
        assert np.array_equal(got[k], ref[k]), k
    # twenty more steps through the graph
    gs.step(20, use_graph=True)
    ctx.check()
    ref = cpu.step(sc, 20, cloud=cloud, state={k: ref[k] for k in STATE})
    got = gs.download()
    for k in STATE:
        assert np.array_equal(got[k], ref[k]), k
    assert np.array_equal(_forces(gs), ref["pforce"])
    gs.close()


def test_cloud_detached_is_the_plain_step(ctx):
    sc = scenes.small_scene(6, nb_side=3, r=1 / 128)
    cloud = random_cloud(12, 8000, 0.25, 0.75)
    gs = api.GpuScene(ctx, sc)
    gs.set_static_cloud(_dev(cloud[0]), _dev(cloud[1]))
    gs.step(3, use_graph=True)
    gs.set_static_cloud(None, None)
    gs.step(4, use_graph=True)
    ctx.check()
    ref = cpu.step(sc, 3, cloud=cloud)
    ref = cpu.step(sc, 4, state={k: ref[k] for k in STATE})
    got = gs.download()
    for k in STATE:
        assert np.array_equal(got[k], ref[k]), k
    assert np.array_equal(_forces(gs), ref["pforce"])
    gs.close()


def test_batch_with_a_cloud_equals_solo(ctx):
    sa = scenes.small_scene(7, nb_side=3, r=1 / 128)
    sb = scenes.small_scene(8, nb_side=3, r=1 / 128)
    cloud = random_cloud(13, 8000, 0.25, 0.75)
    solo = []
    for sc, cl in ((sa, cloud), (sb, None)):
        g = api.GpuScene(ctx, sc)
        if cl is not None:
            g.set_static_cloud(_dev(cl[0]), _dev(cl[1]))
        g.step(12, use_graph=True)
        solo.append(g.download())
        g.close()
    ga, gb = api.GpuScene(ctx, sa), api.GpuScene(ctx, sb)
    ga.set_static_cloud(_dev(cloud[0]), _dev(cloud[1]))
    batch = api.Batch(ctx, [ga, gb])
    base = 1 + 1 + 4 + 1 + 1 + 2
    batch.step(12, use_graph=True)
    ctx.check()
    assert batch.launches_per_step() == base + 1  # the cloud kernel
    for g, want in zip((ga, gb), solo):
        got = g.download()
        for k in STATE:
            assert np.array_equal(got[k], want[k]), k
    # the cloud attached while the scene is in the batch reaches the batch's next step
    ref_b = cpu.step(sb, 12)
    ref_b = cpu.step(sb, 5, cloud=cloud, state={k: ref_b[k] for k in STATE})
    gb.set_static_cloud(_dev(cloud[0]), _dev(cloud[1]))
    batch.step(5, use_graph=True)
    ctx.check()
    got = gb.download()
    for k in STATE:
        assert np.array_equal(got[k], ref_b[k]), k
    batch.close()
    ga.close()
    gb.close()


def test_cloud_argument_errors(ctx):
    sc = scenes.small_scene(9, nb_side=2, r=1 / 128)
    cloud = random_cloud(14, 100, 0.3, 0.7)
    bvh = api.GpuScene(ctx, sc, broadphase="bvh")
    with pytest.raises(ArError):
        bvh.set_static_cloud(_dev(cloud[0]), _dev(cloud[1]))
    bvh.close()
    gs = api.GpuScene(ctx, sc)
    p, n = _dev(cloud[0]), _dev(cloud[1])
    with pytest.raises(ArError):
        call("ar_scene_set_static_cloud", ctx.handle, gs.handle, api.ptr(p), api.ptr(n), -1,
             api.stream_handle())
    with pytest.raises(ArError):
        call("ar_scene_set_static_cloud", ctx.handle, gs.handle, None, api.ptr(n), 100,
             api.stream_handle())
    raw = torch.zeros(401, dtype=torch.float32, device="cuda")
    with pytest.raises(ArError):  # positions not 16-byte aligned
        call("ar_scene_set_static_cloud", ctx.handle, gs.handle, C.c_void_p(raw.data_ptr() + 4),
             api.ptr(n), 100, api.stream_handle())
    gs.close()


def test_depth_image_cloud_in_the_step(ctx):
    """Range image -> cloud and normals on the device -> attached to a scene whose bodies sit
    on the cloud's surface -> steps equal to the oracle's."""
    g = golden("range_image")
    depth, cam = g["depth"], np.ascontiguousarray(g["camera16"], np.float32).reshape(16)
    h, w = depth.shape
    r = 1 / 128
    d_depth = torch.from_numpy(depth.astype(np.int16).view(np.int16).copy()).cuda()
    pos4 = torch.zeros((w * h, 4), dtype=torch.float32, device="cuda")
    radii = torch.zeros(w * h, dtype=torch.float32, device="cuda")
    norm4 = torch.zeros((w * h, 4), dtype=torch.float32, device="cuda")
    call("ar_range_image_cloud", ctx.handle, api.ptr(d_depth), w, h,
         cam.ctypes.data_as(C.c_void_p), C.c_float(r),
         api.ptr(pos4), api.ptr(radii), None, api.stream_handle())
    call("ar_range_image_normals", ctx.handle, api.ptr(pos4), w, h, api.ptr(norm4),
         api.stream_handle())
    # border pixels keep their zero normal; a pixel whose neighbours coincide gets a NaN one
    norm4 = torch.nan_to_num(norm4, nan=0.0, posinf=0.0, neginf=0.0)
    torch.cuda.synchronize()
    cp, cn = pos4.cpu().numpy(), norm4.cpu().numpy()
    unit = np.abs(np.linalg.norm(cn[:, :3], axis=1) - 1.0) < 1e-3
    near = (np.abs(cp[:, :3]).max(1) < 100.0) & unit  # pixels with depth and a normal
    assert near.sum() > 1000
    lo, hi = cp[near, :3].min(0), cp[near, :3].max(0)
    # a scene around the cloud: small cubes placed on surface points, lifted along the normal
    rng = np.random.default_rng(21)
    pick = rng.choice(np.flatnonzero(near), 40, replace=False)
    shape = scenes.cube_body(2, 2 * r)
    centres = cp[pick, :3] + 2.5 * r * cn[pick, :3]
    box_lo, box_hi = lo - 0.1, hi + 0.1
    sc = scenes._assemble([shape] * len(pick), centres, scenes.random_quaternions(rng, len(pick)),
                          rng.normal(0.0, 0.2, (len(pick), 3)), r, box_lo, box_hi,
                          name="cubes on a depth-camera surface")
    gs = api.GpuScene(ctx, sc)
    gs.set_static_cloud(pos4, norm4)
    gs.step(1, use_graph=False)
    gs.step(9, use_graph=True)
    ctx.check()
    ref = cpu.step(sc, 10, cloud=(cp, cn))
    plain = cpu.step(sc, 10)
    got = gs.download()
    for k in STATE:
        assert np.array_equal(got[k], ref[k]), k
    assert not np.array_equal(ref["vel"], plain["vel"])  # the surface pushed the cubes
    gs.close()
