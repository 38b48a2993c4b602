"""Python host interface over the C ABI (device memory and streams come from PyTorch).

``Context`` owns an ar_ctx; ``GpuScene`` is a resident scene stepped with the fused
pipeline; ``Batch`` steps many resident scenes with one launch per stage.  The stage entry
points of include/arsim.h are reachable through ``diploma_thesis_b200._lib.call``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import (AR_BROADPHASE_BVH, AR_BROADPHASE_GRID, SceneDesc, SceneInit, SceneView,
                   SimParams, StepView, call, lib)
from .scenes import Scene


def stream_handle(stream: torch.cuda.Stream | None = None) -> C.c_void_p:
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


class DevicePtr(C.c_void_p):
    """A c_void_p that keeps its tensor alive for as long as the pointer object lives (so an
    argument like ptr(torch.tensor(...)) is not freed, and its memory handed to the next
    allocation, before the call it is passed to)."""


def ptr(t: torch.Tensor | None) -> C.c_void_p:
    if t is None:
        return C.c_void_p(None)
    assert t.is_cuda and t.is_contiguous(), "device tensors must be contiguous CUDA tensors"
    p = DevicePtr(t.data_ptr())
    p.tensor = t
    return p


class Context:
    def __init__(self, device: int = 0):
        torch.cuda.set_device(device)
        torch.cuda.init()
        self.handle = C.c_void_p()
        call("ar_ctx_create", device, C.byref(self.handle))

    def status(self, stream=None) -> int:
        return lib.ar_ctx_status(self.handle, stream_handle(stream))

    def check(self, stream=None) -> None:
        _lib.check(self.status(stream), "ar_ctx_status")

    def close(self) -> None:
        if self.handle:
            lib.ar_ctx_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):  # pragma: no cover - best effort
        try:
            self.close()
        except Exception:
            pass


def broadphase_code(b) -> int:
    """'grid' / 'bvh' (or the AR_BROADPHASE_* value) -> AR_BROADPHASE_*."""
    if isinstance(b, str):
        codes = {"grid": AR_BROADPHASE_GRID, "bvh": AR_BROADPHASE_BVH}
        if b not in codes:
            raise ValueError(f"unknown broad phase {b!r} (grid or bvh)")
        return codes[b]
    if b not in (AR_BROADPHASE_GRID, AR_BROADPHASE_BVH):
        raise ValueError(f"unknown broad phase {b!r}")
    return int(b)


def make_desc(scene: Scene, broadphase: int = AR_BROADPHASE_GRID, block_size: int = 0,
              cell_size: float | None = None, grid_log2=None) -> SceneDesc:
    d = SceneDesc()
    d.num_bodies = scene.num_bodies
    d.num_particles = scene.num_particles
    d.radius = scene.radius
    for a in range(3):
        d.box_min[a] = float(scene.box_min[a])
        d.box_max[a] = float(scene.box_max[a])
        d.gravity[a] = float(scene.gravity[a])
    d.dt = scene.dt
    d.spring = scene.spring
    d.damping = scene.damping
    d.shear = scene.shear
    d.attraction = scene.attraction
    d.broadphase = broadphase
    d.cell_size = scene.cell_size if cell_size is None else cell_size
    g = scene.grid_log2 if grid_log2 is None else grid_log2
    for a in range(3):
        d.grid_log2[a] = int(g[a])
    d.block_size = block_size
    return d


def _np_ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


class GpuScene:
    """A scene resident on the device, advanced by ar_step."""

    def __init__(self, ctx: Context, scene: Scene, block_size: int = 0,
                 cell_size: float | None = None, grid_log2=None, broadphase="grid",
                 stream=None):
        self.ctx = ctx
        self.scene = scene
        self.broadphase = broadphase_code(broadphase)
        self.desc = make_desc(scene, self.broadphase, block_size, cell_size, grid_log2)
        self._keep = [np.ascontiguousarray(a) for a in (
            scene.body_pos, scene.body_quat, scene.body_vel, scene.body_angvel,
            scene.body_mass.astype(np.float32), scene.body_inv_inertia.astype(np.float32),
            scene.body_offsets.astype(np.int32), scene.particle_rel)]
        init = SceneInit(*[_np_ptr(a) for a in self._keep])
        self.handle = C.c_void_p()
        call("ar_scene_create", ctx.handle, C.byref(self.desc), C.byref(init),
             stream_handle(stream), C.byref(self.handle))
        self.num_bodies = scene.num_bodies
        self.num_particles = scene.num_particles

    def step(self, n: int = 1, use_graph: bool = True, stream=None) -> None:
        call("ar_step", self.ctx.handle, self.handle, int(n), int(use_graph),
             stream_handle(stream))

    def download(self) -> dict[str, np.ndarray]:
        nb = self.num_bodies
        out = {k: np.zeros((nb, 4), np.float32) for k in ("pos", "quat", "vel", "angvel")}
        call("ar_scene_download", self.handle, _np_ptr(out["pos"]), _np_ptr(out["quat"]),
             _np_ptr(out["vel"]), _np_ptr(out["angvel"]), stream_handle())
        return out

    def upload(self, pos, quat, vel, angvel, stream=None) -> None:
        """Overwrite body state from (preferably pinned) host arrays, asynchronously."""
        call("ar_scene_upload", self.handle, *[_np_ptr(a) if a is not None else None
                                               for a in (pos, quat, vel, angvel)],
             stream_handle(stream))

    def upload_state(self, state: np.ndarray, stream=None) -> None:
        """Overwrite body state from one (preferably pinned) [4, B, 4] float32 host array:
        pos, quat, vel, angvel; asynchronous, one copy."""
        assert state.dtype == np.float32 and state.size == 16 * self.num_bodies
        assert state.flags.c_contiguous
        call("ar_scene_upload_state", self.handle, _np_ptr(state), stream_handle(stream))

    def download_state(self, state: np.ndarray | None = None, stream=None,
                       wait: bool = True) -> np.ndarray:
        """Body state into a [4, B, 4] float32 host array (pos, quat, vel, angvel) with one
        copy; with wait=False the copy is only queued on `stream` (pinned memory)."""
        if state is None:
            state = np.zeros((4, self.num_bodies, 4), np.float32)
        assert state.dtype == np.float32 and state.size == 16 * self.num_bodies
        assert state.flags.c_contiguous
        call("ar_scene_download_state" if wait else "ar_scene_download_state_async", self.handle,
             _np_ptr(state), stream_handle(stream))
        return state

    def set_static_cloud(self, pos4: torch.Tensor | None, norm4: torch.Tensor | None,
                         stream=None) -> None:
        """Attach a static point cloud (device float32 [M, 4] positions and normals) whose
        points push the particles within 2r from the next step on (ar_scene_set_static_cloud);
        None detaches it."""
        if pos4 is None:
            call("ar_scene_set_static_cloud", self.ctx.handle, self.handle, None, None, 0,
                 stream_handle(stream))
            return
        for t in (pos4, norm4):
            assert t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()
            assert t.dim() == 2 and t.shape[1] == 4
        assert pos4.shape == norm4.shape
        call("ar_scene_set_static_cloud", self.ctx.handle, self.handle, ptr(pos4), ptr(norm4),
             int(pos4.shape[0]), stream_handle(stream))

    def step_io(self, state_in: np.ndarray, n: int, state_out: np.ndarray, stream=None) -> None:
        """Upload the packed state, step n times (graph), copy the packed state back, in one
        call (ar_scene_step_io); both arrays are [4, B, 4] float32 pinned host arrays and may be
        the same."""
        for a in (state_in, state_out):
            assert a.dtype == np.float32 and a.size == 16 * self.num_bodies
            assert a.flags.c_contiguous
        call("ar_scene_step_io", self.ctx.handle, self.handle, _np_ptr(state_in), int(n),
             _np_ptr(state_out), stream_handle(stream))

    def download_into(self, pos, quat, vel, angvel, stream=None) -> None:
        call("ar_scene_download", self.handle, *[_np_ptr(a) if a is not None else None
                                                 for a in (pos, quat, vel, angvel)],
             stream_handle(stream))

    def profile(self, n: int, stream=None) -> list[float]:
        """Average device ms per stage over n eager steps: grid (clear, keys, sort, scatter,
        collide, body); BVH (clear, keys, sort, tree, collide, body)."""
        out = (C.c_float * 6)()
        call("ar_step_profile", self.ctx.handle, self.handle, int(n), out, stream_handle(stream))
        return list(out)

    def view(self) -> SceneView:
        v = SceneView()
        call("ar_scene_get_view", self.handle, C.byref(v))
        return v

    def step_view(self) -> StepView:
        v = StepView()
        call("ar_scene_step_view", self.handle, C.byref(v))
        return v

    def grid_info(self):
        o = (C.c_float * 3)()
        c = (C.c_float * 3)()
        d = (C.c_uint32 * 3)()
        call("ar_scene_grid_info", self.handle, o, c, d)
        return list(o), list(c), list(d)

    def launches_per_step(self) -> int:
        return int(lib.ar_scene_launches_per_step(self.handle))

    def close(self) -> None:
        if self.handle:
            lib.ar_scene_destroy(self.handle)
            self.handle = C.c_void_p()

    def download_async(self, stream=None) -> dict[str, np.ndarray]:
        """Queue a copy of the body state into pinned host arrays on `stream` (no wait); the
        arrays are valid once the stream has reached this point."""
        nb = self.num_bodies
        pinned = {k: torch.empty((nb, 4), dtype=torch.float32, pin_memory=True)
                  for k in ("pos", "quat", "vel", "angvel")}
        out = {k: v.numpy() for k, v in pinned.items()}
        call("ar_scene_download_async", self.handle, *[_np_ptr(out[k]) for k in
                                                       ("pos", "quat", "vel", "angvel")],
             stream_handle(stream))
        out["_pinned"] = pinned  # keeps the pinned blocks alive
        return out

    def model_matrices(self, stream=None) -> torch.Tensor:
        """[B, 4, 4] device tensor of per-body model matrices (glm column-major: row i of the
        tensor is column i of the matrix) for a renderer."""
        out = torch.empty((self.num_bodies, 4, 4), dtype=torch.float32, device="cuda")
        call("ar_scene_model_matrices", self.handle, ptr(out), stream_handle(stream))
        return out

    def close_async(self, stream=None) -> None:
        """Free in stream order on `stream`; every use of the scene must precede that point."""
        if self.handle:
            call("ar_scene_destroy_async", self.handle, stream_handle(stream))
            self.handle = C.c_void_p()


class Batch:
    """Many resident scenes advanced together (one launch per stage, CUDA graph)."""

    def __init__(self, ctx: Context, scenes: list[GpuScene] | None = None):
        self.ctx = ctx
        self.handle = C.c_void_p()
        call("ar_batch_create", ctx.handle, C.byref(self.handle))
        self.scenes: list[GpuScene] = []
        if scenes:
            self.set_scenes(scenes)

    def set_scenes(self, scenes: list[GpuScene], steps_left=None) -> None:
        """Member list; steps_left[i] (optional) caps how many of the following steps integrate
        scene i (it is frozen afterwards)."""
        self.scenes = list(scenes)
        arr = (C.c_void_p * max(1, len(scenes)))(*[s.handle for s in scenes])
        if steps_left is None:
            call("ar_batch_set_scenes", self.handle, arr, len(scenes))
        else:
            lim = np.ascontiguousarray(steps_left, dtype=np.int64)
            assert len(lim) == len(scenes)
            call("ar_batch_set_scenes_limited", self.handle, arr, len(scenes),
                 C.c_void_p(lim.ctypes.data))

    def step(self, n: int = 1, use_graph: bool = True, stream=None) -> None:
        call("ar_batch_step", self.ctx.handle, self.handle, int(n), int(use_graph),
             stream_handle(stream))

    def launches_per_step(self) -> int:
        return int(lib.ar_batch_launches_per_step(self.handle))

    def profile(self, n: int, stream=None) -> list[float]:
        out = (C.c_float * 6)()
        call("ar_batch_profile", self.ctx.handle, self.handle, int(n), out, stream_handle(stream))
        return list(out)

    def close(self) -> None:
        if self.handle:
            lib.ar_batch_destroy(self.handle)
            self.handle = C.c_void_p()


class _DeviceArray:
    """Minimal __cuda_array_interface__ exporter for a raw device address."""

    _TYPESTR = {torch.float32: "<f4", torch.int32: "<i4", torch.int64: "<i8",
                torch.uint8: "|u1", torch.float64: "<f8"}

    def __init__(self, addr: int, count: int, dtype: torch.dtype):
        self.__cuda_array_interface__ = {"shape": (count,), "typestr": self._TYPESTR[dtype],
                                         "data": (int(addr), False), "version": 3,
                                         "strides": None}


def device_view(addr: int, count: int, dtype: torch.dtype, device: int = 0) -> torch.Tensor:
    """Copy `count` elements starting at a raw device address into a new tensor."""
    if count == 0:
        return torch.empty(0, dtype=dtype, device=f"cuda:{device}")
    torch.cuda.synchronize()
    return torch.as_tensor(_DeviceArray(addr, count, dtype), device=f"cuda:{device}").clone()


def sim_params(radius: float, grid_origin, cell, grid_dims, spring=0.5, damping=0.02,
               shear=0.1, attraction=0.0, gravity=(0.0, -9.81, 0.0), w_damping=1.0) -> SimParams:
    p = SimParams()
    p.particle_radius = radius
    for a in range(3):
        p.world_origin[a] = grid_origin[a]
        p.cell_size[a] = cell[a] if np.ndim(cell) else cell
        p.grid_size[a] = int(grid_dims[a])
        p.gravity[a] = gravity[a]
    p.num_cells = int(np.prod(grid_dims))
    p.spring, p.damping, p.shear, p.attraction = spring, damping, shear, attraction
    p.w_damping = w_damping
    p.global_damping = 1.0
    p.boundary_damping = -0.5
    return p
