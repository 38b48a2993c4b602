"""The oracle's sequential-impulse path (CPU): the contact search pinned against the reference's
own FindRigidBodyCollisionsUniformGridKernel (golden fixture tests/golden/sis_find.npz), the
contact gather and the solver pinned against the reference's own host loops (golden fixture
tests/golden/sis_solve.npz, and live where the reference build exists), and the solver against
the reference's known-answer setup and conservation laws."""
from pathlib import Path

import numpy as np
import pytest

from oracle import cpu, ref

GOLDEN = Path(__file__).resolve().parent / "golden"


def test_find_contacts_grid_matches_reference_fixture():
    g = np.load(GOLDEN / "sis_find.npz")
    cd, cb, cp = cpu.find_contacts_grid((0, 0, 0), float(g["cell"]), g["dims"], float(g["radius"]),
                                        g["rb"], g["spos"], g["sidx"], g["cell_start"],
                                        g["cell_end"])
    assert (cd > 0).sum() > 1000
    assert np.array_equal(cd, g["contact_distance"])
    assert np.array_equal(cb, g["contact_body"])
    assert np.array_equal(cp, g["contact_particle"])


def cube_on_ground(iterations=18):
    """simulationTest (Misc/main.cpp:22-98): a cube of side 6 and mass 1 falling at 1 m/s onto
    the ground, four corner contacts with normal +y; the total accumulated impulse is m |v| = 1
    and the cube comes to rest.  (The solver here is SequentialImpulseSolver's, which adds
    friction to one-body contacts, so it takes the reference step's 18 iterations rather than
    the test's 8 to settle within 1e-5.)"""
    side, m = 6.0, 1.0
    inv_i = np.eye(3, dtype=np.float32) * np.float32(6 / (m * side * side))
    r = np.array([[-3, -3, -3], [3, -3, -3], [-3, -3, 3], [3, -3, 3]], np.float32)
    contacts = {"normal": np.tile(np.array([0, 1, 0, 0], np.float32), (4, 1)),
                "point": np.concatenate([r, np.zeros((4, 1), np.float32)], 1),
                "body1": np.zeros(4, np.int32), "body2": np.full(4, -1, np.int32),
                "bias": np.zeros(4, np.float32)}
    cms = np.zeros((1, 4), np.float32)
    vel = np.array([[0, -1, 0, 0]], np.float32)
    ang = np.zeros((1, 4), np.float32)
    return contacts, cms, vel, ang, inv_i.reshape(1, 9), np.array([m], np.float32), iterations


def test_sequential_impulse_cube_on_ground():
    contacts, cms, vel, ang, ib, mass, it = cube_on_ground()
    v, w, acc, f1, f2 = cpu.sequential_impulse(contacts, cms, vel, ang, ib, mass, iterations=it)
    assert abs(float(acc.sum()) - 1.0) < 1e-5
    assert np.abs(v[0, :3]).max() < 1e-5 and np.abs(w[0, :3]).max() < 1e-5
    assert np.all(acc >= 0)


def test_sequential_impulse_conserves_momentum_between_bodies():
    rng = np.random.default_rng(3)
    nb, k = 6, 40
    b1 = rng.integers(0, nb, k).astype(np.int32)
    b2 = ((b1 + rng.integers(1, nb, k)) % nb).astype(np.int32)
    nrm = rng.normal(0, 1, (k, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    cms = np.zeros((nb, 4), np.float32)
    cms[:, :3] = rng.uniform(-1, 1, (nb, 3))
    contacts = {"normal": np.concatenate([nrm, np.zeros((k, 1))], 1).astype(np.float32),
                "point": np.concatenate([rng.uniform(-1, 1, (k, 3)), np.zeros((k, 1))], 1).astype(np.float32),
                "body1": b1, "body2": b2, "bias": rng.normal(0, 0.1, k).astype(np.float32)}
    vel = np.zeros((nb, 4), np.float32)
    vel[:, :3] = rng.normal(0, 1, (nb, 3))
    ang = np.zeros((nb, 4), np.float32)
    mass = rng.uniform(0.5, 2.0, nb).astype(np.float32)
    ib = np.tile(np.eye(3, dtype=np.float32).reshape(9), (nb, 1))
    v, w, acc, _, _ = cpu.sequential_impulse(contacts, cms, vel, ang, ib, mass)
    p0 = (mass[:, None].astype(np.float64) * vel[:, :3]).sum(0)
    p1 = (mass[:, None].astype(np.float64) * v[:, :3]).sum(0)
    assert np.abs(p1 - p0).max() < 1e-4  # body pairs exchange equal and opposite impulses
    assert np.all((acc >= 0) & (acc <= 100))


CONTACT_KEYS = ("normal", "point", "body1", "body2", "bias")


def _sis_golden():
    from conftest import golden
    return golden("sis_solve")


def test_oracle_gather_and_solver_equal_the_reference_host_loops():
    """tests/golden/sis_solve.npz holds the output of the reference's own GatherRigidBodyCollisions,
    GatherAugmentedRealityCollisions and SequentialImpulseSolver (Particles/updateFunctions.cpp:
    1431-1874, built for the host by oracle/ref_build.py).  The oracle's restatement gives the
    same contacts, velocities and accumulated impulses bit for bit, for body-body contacts and
    for the solver's one-body (static scene) branch."""
    z = _sis_golden()
    c = cpu.gather_contacts(float(z["radius"]), float(z["restitution"]), z["rb_idx"], z["cms"],
                            z["vel"], z["ang"], z["rel"], z["contact_distance"],
                            z["contact_body"], z["contact_particle"])
    for key in CONTACT_KEYS:
        assert np.array_equal(c[key], z["rb_" + key]), key
    for tag, contacts in (("rb", c), ("ar", {k: z["ar_" + k] for k in CONTACT_KEYS})):
        v, w, a0, a1, a2 = cpu.sequential_impulse(
            contacts, z["cms"], z["vel"], z["ang"], z["inv_inertia"], z["mass"],
            iterations=int(z["iterations"]), ar_friction=float(z["ar_friction"]),
            rb_friction=float(z["rb_friction"]), gravity_y=float(z["gravity_y"]))
        assert np.array_equal(v, z[tag + "_vel"]) and np.array_equal(w, z[tag + "_ang"]), tag
        acc = z[tag + "_acc"]
        for i, a in enumerate((a0, a1, a2)):
            assert np.array_equal(a, acc[:, i]), (tag, i)
    assert len(z["ar_body1"]) > 100 and (z["ar_body2"] == -1).all()


@pytest.mark.skipif(not ref.available(), reason="reference CPU build not present")
def test_oracle_equals_reference_host_loops_on_fresh_inputs():
    """The same comparison run live against the reference build, on another seeded state and
    with friction and restitution values of its own."""
    z = _sis_golden()
    rng = np.random.default_rng(99)
    nb = len(z["cms"])
    cms = z["cms"].copy()
    cms[:, :3] += rng.normal(0, 0.01, (nb, 3)).astype(np.float32)
    vel = rng.normal(0, 0.5, (nb, 4)).astype(np.float32)
    ang = rng.normal(0, 2, (nb, 4)).astype(np.float32)
    vel[:, 3] = ang[:, 3] = 0
    prm = ref.sim_params(float(z["radius"]), (0, 0, 0), float(z["cell"]), z["dims"],
                         gravity=(0.0, -3.0, 0.0))
    prm.rb_restitution, prm.rb_friction, prm.ar_friction = 0.8, 0.4, 0.2
    r = ref.sis_step(prm, z["rb_idx"], z["offsets"], cms, vel, ang, z["inv_inertia"], z["mass"],
                     z["rel"], z["contact_distance"], z["contact_body"], z["contact_particle"])
    c = cpu.gather_contacts(float(z["radius"]), 0.8, z["rb_idx"], cms, vel, ang, z["rel"],
                            z["contact_distance"], z["contact_body"], z["contact_particle"])
    for key in CONTACT_KEYS:
        assert np.array_equal(c[key], r[key]), key
    v, w, a0, a1, a2 = cpu.sequential_impulse(c, cms, vel, ang, z["inv_inertia"], z["mass"],
                                              iterations=18, ar_friction=0.2, rb_friction=0.4,
                                              gravity_y=-3.0)
    assert np.array_equal(v, r["vel"]) and np.array_equal(w, r["ang"])
    assert np.array_equal(a0, r["acc"][:, 0]) and np.array_equal(a2, r["acc"][:, 2])
