"""The reference's default update path, updateUniformGridSIS (RigidBodies/UniformGridUpdate.cpp
:734-815), run on the device through the C ABI, in REFERENCE semantics.

One step:
  Integrate_Rigid_Body_System_GPU (Particles/updateFunctions.cpp:2899-2944):
      GPUintegratorKernel -> computeGlobalAttributes -> resetQuaternion
  Find_Rigid_Body_Collisions_Uniform_Grid (RigidBodies/UniformGridUpdate.cpp:336-437):
      calcHash -> sort -> reorderDataAndFindCellStart -> contact distances zeroed ->
      FindRigidBodyCollisionsUniformGridKernel
  GatherRigidBodyCollisions + SequentialImpulseSolver (Particles/updateFunctions.cpp:1431-1874,
      host loops in the reference, device kernels here) -> computeGlobalAttributes

Every array stays on the device; the reference copies the body state to the host and back
twice per step.  Body state uses the reference's layouts: float4 centres of mass, velocities
and angular velocities (w = 0), glm::quat rotation of the step (x, y, z, w), glm::mat3 inverse
inertia (body frame) and its world-frame copy, particle offsets from the centre (w = 0).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import api
from ._lib import call
from .api import ptr, stream_handle
from .scenes import Scene

ITERATIONS = 18  # SequentialImpulseSolver's sweeps per step


def _dev(a: np.ndarray, dtype=torch.float32) -> torch.Tensor:
    return torch.from_numpy(np.ascontiguousarray(a)).to(dtype).cuda()


class SISScene:
    """A scene stepped with the sequential-impulse path."""

    def __init__(self, ctx: api.Context, scene: Scene, dt: float, grid_log2=(7, 7, 7),
                 gravity=(0.0, -9.81, 0.0), restitution: float = 1.0, rb_friction: float = 0.1,
                 ar_friction: float = 0.3, w_damping: float = 1.0):
        """gravity is per second: the reference's integrator adds params.gravity to the velocity
        once per step, so it is given gravity * dt."""
        self.ctx = ctx
        self.dt = float(dt)
        self.n, self.nb = scene.num_particles, scene.num_bodies
        dims = tuple(1 << int(g) for g in grid_log2)
        self.num_cells = int(np.prod(dims))
        p = api.sim_params(scene.radius, tuple(float(x) for x in scene.box_min),
                           2 * float(scene.radius), dims,
                           gravity=tuple(float(g) * self.dt for g in gravity), w_damping=w_damping)
        p.rb_restitution, p.rb_friction, p.ar_friction = restitution, rb_friction, ar_friction
        self.params = p
        n, nb = self.n, self.nb
        self.cms = _dev(scene.body_pos * np.array([1, 1, 1, 0], np.float32))
        self.vel = _dev(scene.body_vel * np.array([1, 1, 1, 0], np.float32))
        self.ang = _dev(scene.body_angvel * np.array([1, 1, 1, 0], np.float32))
        self.quat = _dev(np.tile(np.array([0, 0, 0, 1], np.float32), (nb, 1)))
        self.ib = _dev(scene.body_inv_inertia)
        self.cur = torch.zeros((nb, 9), dtype=torch.float32, device="cuda")
        self.mass = _dev(scene.body_mass)
        # particle offsets in the world frame (the reference rotates them in place each step)
        rel = np.zeros((n, 4), np.float32)
        w = scene.world_positions()
        rel[:, :3] = w[:, :3] - scene.body_pos[scene.body_index(), :3]
        self.rel = _dev(rel)
        self.rb = _dev(scene.body_index(), torch.int32)
        self.pos = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
        self.pvel = torch.zeros_like(self.pos)
        z = lambda shape, dt=torch.int32: torch.zeros(shape, dtype=dt, device="cuda")
        self.hash, self.idx, self.shash, self.sidx = z(n), z(n), z(n), z(n)
        self.cstart, self.cend = z(self.num_cells), z(self.num_cells)
        self.spos, self.svel = z((n, 4), torch.float32), z((n, 4), torch.float32)
        self.cdist = z(n, torch.float32)
        self.cbody, self.cpart = z(n), z(n)
        self.normal, self.point = z((n, 4), torch.float32), z((n, 4), torch.float32)
        self.body1, self.body2, self.count = z(n), z(n), z(1)
        self.bias, self.acc0, self.acc1, self.acc2 = (z(n, torch.float32) for _ in range(4))
        # particle positions for the first contact search (identity rotation)
        call("ar_global_attributes", ctx.handle, n, nb, ptr(self.cms), ptr(self.vel),
             ptr(self.ang), ptr(self.quat), ptr(self.rb), ptr(self.rel), ptr(self.pos),
             ptr(self.pvel), stream_handle())

    # -- the two halves of a step ---------------------------------------------------------------
    def integrate(self, stream=None) -> None:
        """Integrate_Rigid_Body_System_GPU: bodies, then particles, then the step rotation
        reset."""
        s, h = stream_handle(stream), self.ctx.handle
        call("ar_integrate_reference", h, C.byref(self.params), self.dt, self.nb, ptr(self.cms),
             ptr(self.vel), ptr(self.ang), ptr(self.quat), ptr(self.ib), ptr(self.cur), None,
             None, ptr(self.mass), s)
        call("ar_global_attributes", h, self.n, self.nb, ptr(self.cms), ptr(self.vel),
             ptr(self.ang), ptr(self.quat), ptr(self.rb), ptr(self.rel), ptr(self.pos),
             ptr(self.pvel), s)
        call("ar_reset_quaternions", h, ptr(self.quat), self.nb, s)

    def solve(self, stream=None) -> None:
        """Contact search, gather, sequential impulses, then particle velocities."""
        s, h, n = stream_handle(stream), self.ctx.handle, self.n
        pp = C.byref(self.params)
        call("ar_calc_hash", h, pp, ptr(self.pos), n, ptr(self.hash), ptr(self.idx), s)
        call("ar_radix_sort_pairs_u32", h, ptr(self.hash), ptr(self.idx), ptr(self.shash),
             ptr(self.sidx), n, 0, 32, s)
        call("ar_reorder_cells", h, ptr(self.shash), ptr(self.sidx), ptr(self.pos),
             ptr(self.pvel), n, self.num_cells, ptr(self.cstart), ptr(self.cend),
             ptr(self.spos), ptr(self.svel), s)
        call("ar_fill_f32", h, ptr(self.cdist), n, 0.0, s)
        call("ar_find_contacts_grid", h, pp, ptr(self.rb), ptr(self.spos), ptr(self.sidx),
             ptr(self.cstart), ptr(self.cend), n, ptr(self.cdist), ptr(self.cbody),
             ptr(self.cpart), s)
        call("ar_gather_contacts", h, pp, n, ptr(self.rb), ptr(self.cms), ptr(self.vel),
             ptr(self.ang), ptr(self.rel), ptr(self.cdist), ptr(self.cbody), ptr(self.cpart), n,
             ptr(self.normal), ptr(self.point), ptr(self.body1), ptr(self.body2),
             ptr(self.bias), ptr(self.acc0), ptr(self.acc1), ptr(self.acc2), ptr(self.count), s)
        call("ar_sequential_impulse", h, pp, ptr(self.count), n, ptr(self.normal),
             ptr(self.point), ptr(self.body1), ptr(self.body2), ptr(self.bias), ptr(self.acc0),
             ptr(self.acc1), ptr(self.acc2), self.nb, ptr(self.cms), ptr(self.vel), ptr(self.ang),
             ptr(self.cur), ptr(self.mass), ITERATIONS, s)
        call("ar_global_attributes", h, n, self.nb, ptr(self.cms), ptr(self.vel), ptr(self.ang),
             ptr(self.quat), ptr(self.rb), ptr(self.rel), ptr(self.pos), ptr(self.pvel), s)

    def step(self, steps: int = 1, stream=None) -> None:
        for _ in range(steps):
            self.integrate(stream)
            self.solve(stream)

    def state(self) -> dict[str, np.ndarray]:
        torch.cuda.synchronize()
        out = {k: getattr(self, k).cpu().numpy() for k in
               ("cms", "vel", "ang", "quat", "cur", "rel", "pos", "pvel")}
        out["contacts"] = int(self.count.cpu().numpy()[0])
        return out
