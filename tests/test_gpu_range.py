"""Depth-camera ingestion on the device (ar_range_image_cloud / ar_range_image_normals) against
the reference's own kernels (golden fixture, bit for bit) and against the oracle on an image
whose size is not a whole number of the reference's 16 x 32 blocks (every pixel covered)."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import golden
from diploma_thesis_b200 import api
from diploma_thesis_b200._lib import call
from oracle import cpu

pytestmark = pytest.mark.gpu


def _run(ctx, depth, camera16, radius):
    h, w = depth.shape
    d = torch.from_numpy(depth.astype(np.int16).view(np.int16).copy()).cuda()
    pos = torch.full((h * w, 4), float("nan"), device="cuda")
    radii = torch.full((h * w,), float("nan"), device="cuda")
    vao = torch.full((h * w, 5), float("nan"), device="cuda")
    norm = torch.full((h * w, 4), float("nan"), device="cuda")
    cam = np.ascontiguousarray(np.asarray(camera16, np.float32).reshape(16))
    call("ar_range_image_cloud", ctx.handle, api.ptr(d), w, h,
         cam.ctypes.data_as(C.c_void_p), C.c_float(radius), api.ptr(pos), api.ptr(radii),
         api.ptr(vao), api.stream_handle())
    call("ar_range_image_normals", ctx.handle, api.ptr(pos), w, h, api.ptr(norm),
         api.stream_handle())
    ctx.check()
    return {k: t.cpu().numpy() for k, t in
            (("pos4", pos), ("radii", radii), ("vao5", vao), ("norm4", norm))}


def _same(a, b):
    written = ~np.isnan(b)
    assert np.array_equal(~np.isnan(a), written)
    assert np.array_equal(a[written].view(np.uint32), b[written].view(np.uint32))


def test_range_image_equals_reference(ctx):
    z = golden("range_image")
    out = _run(ctx, z["depth"], z["camera16"], float(z["radius"]))
    for k in ("pos4", "radii", "vao5", "norm4"):
        _same(out[k], z[k])


def test_range_image_ragged_size_equals_oracle(ctx):
    rng = np.random.default_rng(5)
    h, w = 45, 70  # not whole 16 x 32 blocks
    depth = rng.integers(0, 9000, (h, w)).astype(np.uint16)
    depth[rng.random((h, w)) < 0.05] = 0
    cam = np.eye(4, dtype=np.float32)
    cam[3, :3] = (0.5, 0.25, -1.0)
    out = _run(ctx, depth, cam.reshape(16), 0.01)
    ref = cpu.range_image_cloud(depth, cam.reshape(16), 0.01)
    for k in ("pos4", "radii", "vao5"):
        _same(out[k], ref[k])
    _same(out["norm4"], cpu.range_image_normals(ref["pos4"], w, h))
