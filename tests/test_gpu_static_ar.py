"""The static-scene (augmented-reality) impulse path on the GPU through the C ABI, against the
reference's own kernel bodies (tests/golden/static_scene_ar.npz): ar_collide_static_scene_impulse
(ARcollisionsUniformGridKernel), ar_find_contacts_static_scene (FindAugmentedRealityCollisions-
UniformGridKernel), ar_gather_static_contacts (GatherAugmentedRealityCollisions) and
ar_sequential_impulse on the gathered list (SequentialImpulseSolver); bit for bit."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import golden
from diploma_thesis_b200 import api
from gpu_util import P, S, call, dev, empty, host

pytestmark = pytest.mark.gpu

KEYS = ("normal", "point", "body1", "body2", "bias")


def _params(z):
    prm = api.sim_params(float(z["radius"]), (0, 0, 0), float(z["cell"]), z["dims"])
    prm.ar_restitution = float(z["ar_restitution"])
    prm.ar_friction = float(z["ar_friction"])
    return prm


def test_impulse_variant_matches_reference(ctx):
    z = golden("static_scene_ar")
    n = len(z["spos"])
    prm = _params(z)
    pf, pt = empty((n, 4)), empty((n, 4))
    count, color = empty(n, torch.int32), empty((n, 4))
    call("ar_collide_static_scene_impulse", ctx.handle, C.byref(prm), P(dev(z["rb_idx"])),
         P(dev(z["rel"])), P(dev(z["inertia"])), P(dev(z["mass"])), P(dev(z["scene_radii"])),
         P(dev(z["spos"])), P(dev(z["svel"])), P(dev(z["scene_spos"])), P(dev(z["sidx"])),
         P(dev(z["scene_sidx"])), P(dev(z["scene_cell_start"])), P(dev(z["scene_cell_end"])), n,
         P(pf), P(pt), P(count), None, P(color), S())
    ctx.check()
    assert np.array_equal(host(pf), z["impulse_force"])
    assert np.array_equal(host(pt), z["impulse_torque"])
    assert np.array_equal(host(count), z["impulse_count"])
    assert np.array_equal(host(color), z["impulse_color"])


def test_find_gather_solve_match_reference(ctx):
    z = golden("static_scene_ar")
    n = len(z["spos"])
    prm = _params(z)
    cd = dev(np.zeros(n, np.float32))
    cp = dev(np.full(n, -1, np.int32))
    color = empty((n, 4))
    call("ar_find_contacts_static_scene", ctx.handle, C.byref(prm), P(dev(z["spos"])),
         P(dev(z["scene_spos"])), P(dev(z["sidx"])), P(dev(z["scene_sidx"])),
         P(dev(z["scene_cell_start"])), P(dev(z["scene_cell_end"])), n, P(cd), P(cp), P(color),
         S())
    ctx.check()
    assert np.array_equal(host(cd), z["contact_distance"])
    assert np.array_equal(host(cp), z["contact_point"])
    assert np.array_equal(host(color), z["find_color"])
    cap = n
    out = {"normal": empty((cap, 4)), "point": empty((cap, 4)), "body1": empty(cap, torch.int32),
           "body2": empty(cap, torch.int32), "bias": empty(cap)}
    acc = [empty(cap) for _ in range(3)]
    cnt = empty(1, torch.int32)
    v, w = dev(z["vel"]), dev(z["ang"])
    call("ar_gather_static_contacts", ctx.handle, C.byref(prm), n, P(dev(z["rb_idx"])),
         P(dev(z["cms"])), P(v), P(w), P(dev(z["rel"])), P(dev(z["scene_normals"])), P(cd),
         P(cp), cap, P(out["normal"]), P(out["point"]), P(out["body1"]), P(out["body2"]),
         P(out["bias"]), P(acc[0]), P(acc[1]), P(acc[2]), P(cnt), S())
    ctx.check()
    k = int(host(cnt)[0])
    assert k == len(z["sis_body1"]) > 100
    for key in KEYS:
        assert np.array_equal(host(out[key])[:k], z["sis_" + key]), key
    call("ar_sequential_impulse", ctx.handle, C.byref(prm), P(cnt), k, P(out["normal"]),
         P(out["point"]), P(out["body1"]), P(out["body2"]), P(out["bias"]), P(acc[0]),
         P(acc[1]), P(acc[2]), len(z["cms"]), P(dev(z["cms"])), P(v), P(w), P(dev(z["inertia"])),
         P(dev(z["mass"])), 18, S())
    ctx.check()
    assert np.array_equal(host(v), z["sis_vel"]) and np.array_equal(host(w), z["sis_ang"])
    for i in range(3):
        assert np.array_equal(host(acc[i])[:k], z["sis_acc"][:, i])


def test_gather_overflow_is_reported(ctx):
    z = golden("static_scene_ar")
    n = len(z["spos"])
    prm = _params(z)
    bufs = [empty((8, 4)), empty((8, 4)), empty(8, torch.int32), empty(8, torch.int32), empty(8),
            empty(8), empty(8), empty(8)]
    cnt = empty(1, torch.int32)
    call("ar_gather_static_contacts", ctx.handle, C.byref(prm), n, P(dev(z["rb_idx"])),
         P(dev(z["cms"])), P(dev(z["vel"])), P(dev(z["ang"])), P(dev(z["rel"])),
         P(dev(z["scene_normals"])), P(dev(z["contact_distance"])), P(dev(z["contact_point"])), 8,
         *[P(b) for b in bufs], P(cnt), S())
    assert ctx.status() == 7  # AR_ERR_OVERFLOW
    assert int(host(cnt)[0]) == len(z["sis_body1"])


def test_bvh_static_variants_match_reference(ctx):
    z = golden("static_scene_bvh")
    n, m = len(z["pos"]), len(z["cms"])
    prm = api.sim_params(float(z["radius"]), (0, 0, 0), 1.0, (4, 4, 4),
                         *[float(x) for x in z["prm"]])
    tree = [P(dev(z[k])) for k in ("is_leaf", "left", "right")]
    scene = [P(dev(z["cms"])), P(dev(z["bounds"]))]
    pf, pt, color = empty((n, 4)), empty((n, 4)), empty((n, 4))
    vel = dev(z["vel"])
    call("ar_collide_bvh_static", ctx.handle, C.byref(prm), P(dev(z["rb_idx"])), P(dev(z["rel"])),
         P(dev(z["pos"])), P(vel), *tree, None, *scene, P(dev(z["radii"])), m, n, P(pf), P(pt),
         P(color), S())
    ctx.check()
    body = z["rb_idx"] >= 0
    assert np.array_equal(host(pf)[body], z["body_force"][body])
    assert np.array_equal(host(pt)[body], z["body_torque"][body])
    assert np.array_equal(host(vel), z["vel_out"]) and np.array_equal(host(color), z["color"])
    cd, cp, fc = dev(np.zeros(n, np.float32)), dev(np.full(n, -1, np.int32)), empty((n, 4))
    call("ar_find_contacts_bvh_static", ctx.handle, C.byref(prm), P(dev(z["pos"])), *tree, None,
         *scene, P(dev(z["sorted_idx"])), P(dev(z["radii"])), m, n, P(cd), P(cp), P(fc), S())
    ctx.check()
    assert np.array_equal(host(cd), z["contact_distance"])
    assert np.array_equal(host(cp), z["contact_point"])
    assert np.array_equal(host(fc), z["find_color"])
