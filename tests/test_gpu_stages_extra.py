"""CUDA entry points for the momentum integrator, free-particle integrator, collideD variant,
ReduceRigidBodyVariables and reference-signature BVH traversal (no parent array), against
the golden fixtures from the reference's kernel bodies and the oracle."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import golden
from diploma_thesis_b200 import api
from gpu_util import F3, P, S, call, dev, empty, host
from oracle import cpu

pytestmark = pytest.mark.gpu


def test_integrate_momentum_golden(ctx):
    g = golden("reference_extra")
    keys = ("cms", "vel", "force", "ang", "quat", "torque", "angmom", "linmom")
    t = {k: dev(g[f"mom_in_{k}"]) for k in keys}
    nb = len(g["mom_in_cms"])
    cur, acc = empty((nb, 9)), empty((nb, 3))
    prm = api.sim_params(1 / 64, (0, 0, 0), 1.0, (1, 1, 1), gravity=(0, -0.5, 0))
    prm.boundary_damping = -0.5
    prm.global_damping = 0.999
    call("ar_integrate_momentum", ctx.handle, C.byref(prm), C.c_float(g["mom_dt"]), nb,
         *[P(t[k]) for k in keys], P(dev(g["mom_in_ib"])), P(cur), P(acc),
         P(dev(g["mom_radii"])), P(dev(g["mom_inv_mass"])), F3(0, 0, 0), F3(1, 1, 1), S())
    for k in keys:
        assert np.array_equal(host(t[k]), g[f"mom_out_{k}"]), k
    assert np.array_equal(host(cur), g["mom_out_cur"])
    assert np.array_equal(host(acc), g["mom_out_acc"])


def test_integrate_particles_golden(ctx):
    g = golden("reference_extra")
    pos, vel = dev(g["fp_pos"]), dev(g["fp_vel"])
    prm = api.sim_params(1 / 64, (0, 0, 0), 1.0, (1, 1, 1), gravity=(0, -0.5, 0))
    prm.boundary_damping = -0.5
    prm.global_damping = 0.999
    call("ar_integrate_particles", ctx.handle, C.byref(prm), C.c_float(0.01), P(pos), P(vel),
         P(dev(g["fp_rb"])), len(g["fp_pos"]), F3(0, 0, 0), F3(1, 1, 1), S())
    assert np.array_equal(host(pos), g["fp_pos_out"])
    assert np.array_equal(host(vel), g["fp_vel_out"])


def test_collide_particles_golden(ctx):
    g = golden("reference_extra")
    d = golden("dem_small")
    n = len(d["pos"])
    prm = api.sim_params(float(d["radius"]), (0, 0, 0), float(d["cell"]), d["dims"],
                         *[float(x) for x in d["prm"]])
    pf, pt, nv = empty((n, 4)), empty((n, 4)), empty((n, 4))
    call("ar_collide_grid_particles", ctx.handle, C.byref(prm), P(dev(g["cd_rb"])),
         P(dev(d["spos"])), P(dev(d["svel"])), P(dev(d["rel"])), P(dev(d["sidx"])),
         P(dev(d["cell_start"])), P(dev(d["cell_end"])), n, P(pf), P(pt), P(nv), S())
    assert np.array_equal(host(pf), g["cd_pforce"])
    assert np.array_equal(host(pt), g["cd_ptorque"])
    assert np.array_equal(host(nv), g["cd_newvel"])


def test_reduce_rigid_body_variables(ctx):
    rng = np.random.default_rng(4)
    pf = rng.normal(0, 1, (3000, 4)).astype(np.float32)
    pt = rng.normal(0, 1, (3000, 4)).astype(np.float32)
    counts = rng.integers(1, 60, 60).astype(np.int32)
    starts = np.concatenate([[0], np.cumsum(counts + 3)[:-1]]).astype(np.int32)  # gaps
    bf0 = rng.normal(0, 1, (60, 4)).astype(np.float32)
    bt0 = rng.normal(0, 1, (60, 4)).astype(np.float32)
    bf, bt = dev(bf0), dev(bt0)
    call("ar_reduce_rigid_body_variables", ctx.handle, P(dev(pf)), P(dev(pt)), P(dev(starts)),
         P(dev(counts)), 60, P(bf), P(bt), S())
    assert ctx.status() == 0
    rf, rt, ok = cpu.reduce_rigid_body_variables(pf, pt, starts, counts, bf0, bt0)
    assert np.array_equal(host(bf), rf) and np.array_equal(host(bt), rt)
    pf[starts[7] + 0, 0] = np.inf
    call("ar_reduce_rigid_body_variables", ctx.handle, P(dev(pf)), P(dev(pt)), P(dev(starts)),
         P(dev(counts)), 60, P(bf), P(bt), S())
    assert ctx.status() == 4  # AR_ERR_NAN


def test_bvh_traversal_without_parent_array(ctx):
    """The reference's traversal wrappers pass no parent links; they are derived."""
    from test_gpu_stages import _golden_tree_on_gpu
    d = golden("dem_small")
    n = len(d["pos"])
    t, sidx, cms, bounds, radii = _golden_tree_on_gpu(ctx, d)
    prm = api.sim_params(float(d["radius"]), (0, 0, 0), float(d["cell"]), d["dims"],
                         *[float(x) for x in d["prm"]])
    pf, pt, pp = empty((n, 4)), empty((n, 4)), empty((n, 4))
    call("ar_collide_bvh_dem", ctx.handle, C.byref(prm), P(dev(d["rb"])), P(dev(d["rel"])),
         P(dev(d["vel"])), P(t["is_leaf"]), P(t["left"]), P(t["right"]), None, P(cms),
         P(bounds), P(sidx), P(radii), n, P(pf), P(pt), P(pp), S())
    assert np.array_equal(host(pf), d["bvh_pforce"])
    assert np.array_equal(host(pt), d["bvh_ptorque"])


def test_static_scene_collisions_golden(ctx):
    """AR static scene: the reference kernel's impulses, angular impulses and colours."""
    g = golden("static_scene")
    n = len(g["spos"])
    prm = api.sim_params(float(g["radius"]), (0, 0, 0), float(g["cell"]), g["dims"],
                         *[float(x) for x in g["prm"]])
    lin, ang = dev(g["lin0"]), dev(g["ang0"])
    color = empty((n, 4))
    call("ar_collide_static_scene_dem", ctx.handle, C.byref(prm), P(dev(g["spos"])),
         P(dev(g["svel"])), P(dev(g["rel"])), P(dev(g["scene_spos"])),
         P(dev(g["scene_normals"])), P(dev(g["sidx"])), P(dev(g["scene_sidx"])),
         P(dev(g["scene_cell_start"])), P(dev(g["scene_cell_end"])), n, P(lin), P(ang),
         P(color), S())
    ctx.check()
    assert np.array_equal(host(lin), g["lin"]) and np.array_equal(host(ang), g["ang"])
    assert np.array_equal(host(color), g["color"])
