"""The reference's own updateUniformGridDEM step (RigidBodies/UniformGridUpdate.cpp:939-999)
and its BVH form, made of the reference's kernel bodies built for the host
(oracle/_ref/libref_cpu.so), plus the same step's state in the reference's layout for the
reference's GPU build (oracle/ref_gpu.py).

BASELINE / TEST INFRASTRUCTURE ONLY: the CPU baseline of bench.py and the checker of the
reference GPU build; the product never imports this module.
"""
from __future__ import annotations

import numpy as np


def reference_layout(scene, grid):
    """The scene in the reference's layout and units: SimParams with the per-step (impulse)
    form of the physical constants (force * dt, velocity increment g * dt), body state as
    float4, the per-step quaternion at the identity and the cumulative one at the scene's
    orientation, world-frame particle offsets (the reference re-rotates them every step), body
    index per particle and particles per body."""
    from oracle import ref
    from diploma_thesis_b200.scenes import quat_to_matrix
    origin, cell, dims = grid
    dt = scene.dt
    prm = ref.sim_params(scene.radius, origin, cell[0], dims, scene.spring * dt,
                         scene.damping * dt, scene.shear * dt, scene.attraction * dt,
                         gravity=tuple(g * dt for g in scene.gravity), w_damping=1.0)
    n, nb = scene.num_particles, scene.num_bodies
    rb = scene.body_index()
    R = quat_to_matrix(scene.body_quat.astype(np.float64))[rb]
    rel = np.zeros((n, 4), np.float32)
    rel[:, :3] = np.einsum("nij,nj->ni", R, scene.particle_rel[:, :3])
    return {"prm": prm, "dt": dt, "ncell": int(np.prod(dims)), "rb": rb.astype(np.int32),
            "counts": np.diff(scene.body_offsets).astype(np.int32), "rel": rel,
            "cms": scene.body_pos.copy(), "vel": scene.body_vel.copy(),
            "ang": scene.body_angvel.copy(),
            "quat": np.tile([0, 0, 0, 1.0], (nb, 1)).astype(np.float32),
            "ib": scene.body_inv_inertia.copy(), "cum": scene.body_quat.copy(),
            "mass": scene.body_mass.copy()}


class ReferenceCPUStep:
    """One updateUniformGridDEM step (RigidBodies/UniformGridUpdate.cpp:939-999) made of the
    reference's own kernel bodies run on the host cores: GPUintegratorKernel,
    computeGlobalAttributes, calcHashD, the CUB-order stable sort, reorder (with its
    full-grid clear), FindAndHandleRigidBodyCollisionsUniformGridKernel and
    ReducePerParticleImpulses.  Physical constants are given the reference's per-step form
    (impulse = force * dt, velocity increment g * dt)."""

    def __init__(self, scene, grid):
        from oracle import ref
        self.ref = ref
        self.s = scene
        L = reference_layout(scene, grid)
        self.prm, self.ncell, self.rb, self.counts, self.rel = (L[k] for k in (
            "prm", "ncell", "rb", "counts", "rel"))
        nb = scene.num_bodies
        self.st = {"cms": L["cms"], "vel": L["vel"], "ang": L["ang"], "quat": L["quat"],
                   "ib": L["ib"], "cur": np.zeros((nb, 9), np.float32),
                   "model": np.zeros((nb, 16), np.float32), "cum": L["cum"]}

    def step(self):
        ref, s = self.ref, self.s
        self.st = ref.gpu_integrator(self.prm, s.dt, self.st)
        self.rel, pos, vel, q = ref.global_attributes(self.st["cms"], self.st["vel"],
                                                      self.st["ang"], self.st["quat"], self.rb,
                                                      self.rel)
        self.st["quat"] = q
        h, idx = ref.calc_hash(self.prm, pos)
        sh, si = ref.sort_pairs_u32(h, idx)
        cs, ce, sp, sv = ref.reorder(sh, si, pos, vel, self.ncell)
        pf, pt = ref.collide_grid_dem(self.prm, self.rb, sp, sv, self.rel, si, cs, ce)
        self.st["vel"], self.st["ang"] = ref.reduce_impulses(
            pf, pt, self.st["vel"], self.st["ang"], s.body_mass, s.body_inv_inertia, self.counts)


class ReferenceCPUStepBVH(ReferenceCPUStep):
    """The BVH form of the same step, from the reference's own kernel bodies on the host cores:
    GPUintegratorKernel, computeGlobalAttributes, findAABBCub, generateMortonCodes, the
    CUB-order stable sort, kernelConstructRadixTreeSoA, kernelConstructLeafNodesSoA,
    kernelConstructInternalNodesSoA, collideBVHSoARigidBody and ReducePerParticleImpulses."""

    def step(self):
        ref, s = self.ref, self.s
        self.st = ref.gpu_integrator(self.prm, s.dt, self.st)
        self.rel, pos, vel, q = ref.global_attributes(self.st["cms"], self.st["vel"],
                                                      self.st["ang"], self.st["quat"], self.rb,
                                                      self.rel)
        self.st["quat"] = q
        mn, mx = ref.aabb(pos)
        codes, idx = ref.morton30(pos, mn, mx)
        sk, si = ref.sort_pairs_u32(codes, idx)
        tree = ref.radix_tree(sk)
        cms, _, bounds, radii = ref.leaves_and_refit(tree, si, pos, s.radius)
        pf, pt, _ = ref.collide_bvh_rigid(self.prm, self.rb, self.rel, vel, tree, cms, bounds, si,
                                          radii)
        self.st["vel"], self.st["ang"] = ref.reduce_impulses(
            pf, pt, self.st["vel"], self.st["ang"], s.body_mass, s.body_inv_inertia, self.counts)


REFERENCE_SEMANTICS = ("the reference's own step (REFERENCE semantics: DEM impulses applied as "
                       "velocity increments, gravity added once per step, world-frame particle "
                       "offsets re-rotated every step); the GPU arm runs the PHYSICAL step of the "
                       "same pipeline (same broad phase, contact law and summation order)")
