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
