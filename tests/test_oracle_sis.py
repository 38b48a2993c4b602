"""The oracle's sequential-impulse path (CPU): the contact search pinned against the reference's
own FindRigidBodyCollisionsUniformGridKernel (golden fixture tests/golden/sis_find.npz), and the
solver against the reference's known-answer setup and conservation laws."""
from pathlib import Path

import numpy as np

from oracle import cpu

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
