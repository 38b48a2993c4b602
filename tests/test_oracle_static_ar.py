"""The oracle's static-scene (augmented-reality) impulse path against the reference's own
kernel bodies (golden fixture tests/golden/static_scene_ar.npz, from oracle/_ref):
ARcollisionsUniformGridKernel (Baraff impulses, own cell examined 27 times),
FindAugmentedRealityCollisionsUniformGridKernel (deepest contact per particle) and
GatherAugmentedRealityCollisions + SequentialImpulseSolver; bit for bit."""
import numpy as np

from conftest import golden
from oracle import cpu

KEYS = ("normal", "point", "body1", "body2", "bias")


def test_impulse_variant_equals_reference():
    z = golden("static_scene_ar")
    pf, pt, count, color, _ = cpu.ar_collide_impulse(
        (0, 0, 0), float(z["cell"]), z["dims"], float(z["radius"]), float(z["ar_restitution"]),
        z["rb_idx"], z["rel"], z["inertia"], z["mass"], z["scene_radii"], z["spos"], z["svel"],
        z["scene_spos"], z["sidx"], z["scene_sidx"], z["scene_cell_start"], z["scene_cell_end"])
    assert (np.abs(z["impulse_force"]).sum(1) > 0).sum() > 100
    assert np.array_equal(pf, z["impulse_force"]) and np.array_equal(pt, z["impulse_torque"])
    assert np.array_equal(count, z["impulse_count"])
    assert np.array_equal(color, z["impulse_color"])
    assert count.max() % 27 == 0  # every impulse is counted once per neighbour iteration


def test_find_gather_solve_equal_reference():
    z = golden("static_scene_ar")
    n = len(z["spos"])
    cd, cp, color = cpu.ar_find_contacts((0, 0, 0), float(z["cell"]), z["dims"],
                                         float(z["radius"]), z["spos"], z["scene_spos"],
                                         z["sidx"], z["scene_sidx"], z["scene_cell_start"],
                                         z["scene_cell_end"], np.zeros(n, np.float32),
                                         np.full(n, -1, np.int32))
    assert np.array_equal(cd, z["contact_distance"]) and np.array_equal(cp, z["contact_point"])
    assert np.array_equal(color, z["find_color"])
    c = cpu.gather_static_contacts(float(z["ar_restitution"]), z["rb_idx"], z["cms"], z["vel"],
                                   z["ang"], z["rel"], z["scene_normals"], cd, cp)
    for key in KEYS:
        assert np.array_equal(c[key], z["sis_" + key]), key
    v, w, a0, a1, a2 = cpu.sequential_impulse(c, z["cms"], z["vel"], z["ang"], z["inertia"],
                                              z["mass"], iterations=18,
                                              ar_friction=float(z["ar_friction"]),
                                              rb_friction=0.0, gravity_y=-9.81)
    assert np.array_equal(v, z["sis_vel"]) and np.array_equal(w, z["sis_ang"])
    assert np.array_equal(a0, z["sis_acc"][:, 0]) and np.array_equal(a2, z["sis_acc"][:, 2])


def _tree(z):
    return {k: z[k] for k in ("is_leaf", "left", "right")}


def test_bvh_static_variants_equal_reference():
    """staticCollideBVHSoARigidBody and FindAugmentedRealityCollisionsBVHKernel (golden fixture
    tests/golden/static_scene_bvh.npz: one particle per body, so the reference's per-body totals
    are the per-particle values; some free particles)."""
    z = golden("static_scene_bvh")
    n = len(z["pos"])
    pf, pt, vel, color = cpu.collide_bvh_static(z["prm"], float(z["radius"]), z["rb_idx"],
                                                z["rel"], z["pos"], z["vel"], _tree(z), z["cms"],
                                                z["bounds"], z["radii"])
    body = z["rb_idx"] >= 0
    assert (np.abs(z["body_force"]).sum(1) > 0).sum() > 100 and (~body).sum() > 10
    assert np.array_equal(pf[body], z["body_force"][body])
    assert np.array_equal(pt[body], z["body_torque"][body])
    assert np.array_equal(vel, z["vel_out"]) and np.array_equal(color, z["color"])
    cd, cp, fc = cpu.find_contacts_bvh_static(float(z["radius"]), z["pos"], _tree(z), z["cms"],
                                              z["bounds"], z["sorted_idx"], z["radii"],
                                              np.zeros(n, np.float32), np.full(n, -1, np.int32))
    assert (cd > 0).sum() > 100
    assert np.array_equal(cd, z["contact_distance"]) and np.array_equal(cp, z["contact_point"])
    assert np.array_equal(fc, z["find_color"])
