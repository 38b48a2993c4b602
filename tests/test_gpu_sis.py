"""The sequential-impulse path on the GPU (ar_find_contacts_grid, ar_gather_contacts,
ar_sequential_impulse) against the reference's contact search (golden fixture) and the oracle's
restatement of the reference's host loops, bit for bit."""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest
import torch

from diploma_thesis_b200 import api
from gpu_util import P, S, call, dev, empty, host
from oracle import cpu
from test_oracle_sis import cube_on_ground

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def _find(ctx, g):
    n = len(g["spos"])
    prm = api.sim_params(float(g["radius"]), (0, 0, 0), float(g["cell"]), g["dims"])
    cd, cb, cp = empty(n), empty(n, torch.int32), empty(n, torch.int32)
    call("ar_find_contacts_grid", ctx.handle, C.byref(prm), P(dev(g["rb"])), P(dev(g["spos"])),
         P(dev(g["sidx"])), P(dev(g["cell_start"])), P(dev(g["cell_end"])), n, P(cd), P(cb),
         P(cp), S())
    ctx.check()
    return host(cd), host(cb), host(cp)


def test_find_contacts_grid_matches_reference(ctx):
    g = np.load(GOLDEN / "sis_find.npz")
    cd, cb, cp = _find(ctx, g)
    assert np.array_equal(cd, g["contact_distance"])
    assert np.array_equal(cb, g["contact_body"])
    assert np.array_equal(cp, g["contact_particle"])


def _gather_inputs(seed=1):
    g = np.load(GOLDEN / "sis_find.npz")
    d = np.load(GOLDEN / "dem_small.npz")
    rng = np.random.default_rng(seed)
    nb = len(d["offsets"]) - 1
    cms = np.zeros((nb, 4), np.float32)
    cms[:, :3] = rng.uniform(0.2, 0.8, (nb, 3))
    vel = rng.normal(0, 1, (nb, 4)).astype(np.float32)
    ang = rng.normal(0, 1, (nb, 4)).astype(np.float32)
    vel[:, 3] = ang[:, 3] = 0
    rel = d["rel"].copy()
    rel[:, 3] = 0
    return g, d, cms, vel, ang, rel


def _gather_gpu(ctx, g, d, cms, vel, ang, rel, capacity):
    n = len(g["rb"])
    prm = api.sim_params(float(g["radius"]), (0, 0, 0), float(g["cell"]), g["dims"])
    prm.rb_restitution = 0.5
    out = {"normal": empty((capacity, 4)), "point": empty((capacity, 4)),
           "body1": empty(capacity, torch.int32), "body2": empty(capacity, torch.int32),
           "bias": empty(capacity), "acc0": empty(capacity), "acc1": empty(capacity),
           "acc2": empty(capacity)}
    cnt = empty(1, torch.int32)
    call("ar_gather_contacts", ctx.handle, C.byref(prm), n, P(dev(g["rb"])), P(dev(cms)),
         P(dev(vel)), P(dev(ang)), P(dev(rel)), P(dev(g["contact_distance"])),
         P(dev(g["contact_body"])), P(dev(g["contact_particle"])), capacity, P(out["normal"]),
         P(out["point"]), P(out["body1"]), P(out["body2"]), P(out["bias"]), P(out["acc0"]),
         P(out["acc1"]), P(out["acc2"]), P(cnt), S())
    return out, cnt, prm


def test_gather_contacts_matches_oracle(ctx):
    g, d, cms, vel, ang, rel = _gather_inputs()
    out, cnt, _ = _gather_gpu(ctx, g, d, cms, vel, ang, rel, len(g["rb"]))
    ctx.check()
    ref = cpu.gather_contacts(float(g["radius"]), 0.5, g["rb"], cms, vel, ang, rel,
                              g["contact_distance"], g["contact_body"], g["contact_particle"])
    k = int(host(cnt)[0])
    assert k == len(ref["body1"]) > 1000
    for key in ("normal", "point", "body1", "body2", "bias"):
        assert np.array_equal(host(out[key])[:k], ref[key]), key
    assert not host(out["acc0"])[:k].any()


def test_gather_overflow_is_reported(ctx):
    g, d, cms, vel, ang, rel = _gather_inputs()
    _, cnt, _ = _gather_gpu(ctx, g, d, cms, vel, ang, rel, 100)
    assert ctx.status() == 7  # AR_ERR_OVERFLOW
    assert int(host(cnt)[0]) > 100


def _solve_gpu(ctx, contacts, cms, vel, ang, ib, mass, iterations, prm=None):
    k = len(contacts["body1"])
    if prm is None:
        prm = api.sim_params(0.01, (0, 0, 0), 0.02, (4, 4, 4))
    prm.ar_friction, prm.rb_friction = 0.3, 0.1
    t = {key: dev(v) for key, v in contacts.items()}
    acc = [empty(k) for _ in range(3)]
    v, w = dev(vel), dev(ang)
    cnt = dev(np.array([k], np.int32))
    call("ar_sequential_impulse", ctx.handle, C.byref(prm), P(cnt), k, P(t["normal"]),
         P(t["point"]), P(t["body1"]), P(t["body2"]), P(t["bias"]), P(acc[0]), P(acc[1]),
         P(acc[2]), len(cms), P(dev(cms)), P(v), P(w), P(dev(ib)), P(dev(mass)), iterations, S())
    ctx.check()
    return host(v), host(w), [host(a) for a in acc]


def test_sequential_impulse_matches_oracle(ctx):
    """Contacts of a packed scene (bodies with many contacts each, so the dependency levels are
    deep) plus one-body contacts: GPU level-by-level solve == the sequential loop."""
    g, d, cms, vel, ang, rel = _gather_inputs(seed=2)
    contacts = cpu.gather_contacts(float(g["radius"]), 0.5, g["rb"], cms, vel, ang, rel,
                                   g["contact_distance"], g["contact_body"],
                                   g["contact_particle"])
    rng = np.random.default_rng(7)
    m = 300  # one-body contacts (body2 = -1) spread through the list
    nrm = rng.normal(0, 1, (m, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    extra = {"normal": np.concatenate([nrm, np.zeros((m, 1))], 1).astype(np.float32),
             "point": contacts["point"][rng.integers(0, len(contacts["point"]), m)],
             "body1": rng.integers(0, len(cms), m).astype(np.int32),
             "body2": np.full(m, -1, np.int32), "bias": rng.normal(0, 0.1, m).astype(np.float32)}
    order = rng.permutation(len(contacts["body1"]) + m)
    allc = {key: np.concatenate([contacts[key], extra[key]])[order] for key in contacts}
    nb = len(cms)
    ib = d["body_inv_inertia"].astype(np.float32)
    mass = d["body_mass"].astype(np.float32)
    gv, gw, gacc = _solve_gpu(ctx, allc, cms, vel, ang, ib, mass, 18)
    rv, rw, a0, a1, a2 = cpu.sequential_impulse(allc, cms, vel, ang, ib, mass, iterations=18)
    assert np.array_equal(gv, rv) and np.array_equal(gw, rw)
    for got, want in zip(gacc, (a0, a1, a2)):
        assert np.array_equal(got, want)
    assert np.abs(rv - vel).max() > 1e-3  # the impulses did something


def _synthetic_contacts(rng, nb, pairs):
    """Random bodies and one contact per (body1, body2) pair (body2 = -1: a one-body contact)."""
    k = len(pairs)
    cms = np.zeros((nb, 4), np.float32)
    cms[:, :3] = rng.uniform(0, 1, (nb, 3))
    vel = np.zeros((nb, 4), np.float32)
    vel[:, :3] = rng.normal(0, 0.1, (nb, 3))
    ang = np.zeros((nb, 4), np.float32)
    ang[:, :3] = rng.normal(0, 0.5, (nb, 3))
    ib = np.zeros((nb, 9), np.float32)
    ib[:, [0, 4, 8]] = rng.uniform(10, 100, (nb, 3))
    mass = rng.uniform(0.5, 2, nb).astype(np.float32)
    b1 = np.array([a for a, _ in pairs], np.int32).reshape(k)
    b2 = np.array([b for _, b in pairs], np.int32).reshape(k)
    nrm = rng.normal(0, 1, (k, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    point = np.zeros((k, 4), np.float32)
    point[:, :3] = cms[b1, :3] + rng.normal(0, 0.01, (k, 3))
    contacts = {"normal": np.concatenate([nrm, np.zeros((k, 1))], 1).astype(np.float32),
                "point": point, "body1": b1, "body2": b2,
                "bias": rng.normal(0, 0.05, k).astype(np.float32)}
    return contacts, cms, vel, ang, ib, mass


def _schedule_case(name, rng):
    if name == "disjoint":  # 1,200 contacts in one level: more than one per thread
        return 2400, [(2 * i, 2 * i + 1) for i in range(1200)]
    if name == "chain":  # few bodies, long dependency chains, one-body contacts among them
        pairs = []
        for i in range(120):
            pairs += [(0, 1), (1, 2)] + ([(0, -1)] if i % 3 == 0 else [])
        return 3, pairs
    if name in ("random", "runs"):  # random bodies; "runs" groups them by first body
        b1 = rng.integers(0, 300, 4000)
        b2 = (b1 + rng.integers(1, 300, 4000)) % 300
        b2[rng.random(4000) < 0.1] = -1
        pairs = list(zip(b1.tolist(), b2.tolist()))
        return 300, sorted(pairs, key=lambda p: p[0]) if name == "runs" else pairs
    return 2, [(0, 1)]  # "single": one level


@pytest.mark.parametrize("name,iterations", [("disjoint", 3), ("chain", 5), ("random", 7),
                                             ("runs", 2), ("runs", 18), ("single", 1),
                                             ("single", 4)])
def test_sequential_impulse_schedules(ctx, name, iterations):
    """Contact lists that stress the solver's schedule (one level wider than the block, long
    chains, random order, runs on one body, a single contact): the overlapped sweeps equal the
    sequential loop bit for bit."""
    rng = np.random.default_rng(sum(name.encode()))
    nb, pairs = _schedule_case(name, rng)
    contacts, cms, vel, ang, ib, mass = _synthetic_contacts(rng, nb, pairs)
    gv, gw, gacc = _solve_gpu(ctx, contacts, cms, vel, ang, ib, mass, iterations)
    rv, rw, a0, a1, a2 = cpu.sequential_impulse(contacts, cms, vel, ang, ib, mass,
                                                iterations=iterations)
    assert np.array_equal(gv, rv) and np.array_equal(gw, rw)
    for got, want in zip(gacc, (a0, a1, a2)):
        assert np.array_equal(got, want)
    assert np.abs(rv - vel).max() > 0


def test_sequential_impulse_cube_on_ground(ctx):
    contacts, cms, vel, ang, ib, mass, it = cube_on_ground()
    v, w, acc = _solve_gpu(ctx, contacts, cms, vel, ang, ib, mass, it)
    rv, rw, a0, _, _ = cpu.sequential_impulse(contacts, cms, vel, ang, ib, mass, iterations=it)
    assert np.array_equal(v, rv) and np.array_equal(acc[0], a0)
    assert abs(float(acc[0].sum()) - 1.0) < 1e-5


def test_sis_steps_match_oracle(ctx):
    """Steps of the sequential-impulse path: after each step's integration the device state is
    snapshotted and the rest of the step (search, gather, solver, particle update) is run by
    the oracle from it; the device's results must equal it bit for bit.  (The integration's
    cosf / sinf are checked on their own, to 1e-5 relative.)"""
    from diploma_thesis_b200 import scenes
    from diploma_thesis_b200.sis import SISScene, ITERATIONS
    sc = scenes.small_scene(4, nb_side=4, packed=True, r=1 / 128)
    g = SISScene(ctx, sc, dt=1e-3, grid_log2=(5, 5, 5))
    rb = sc.body_index()
    dims = (32, 32, 32)
    total = 0
    for _ in range(4):
        g.integrate()
        before = g.state()
        before["mass"] = sc.body_mass.astype(np.float32)
        g.solve()
        ctx.check()
        after = g.state()
        ref = cpu.sis_solve(before, rb, tuple(sc.box_min), 2 * np.float32(sc.radius), dims,
                            sc.radius, gravity_y=g.params.gravity[1], iterations=ITERATIONS)
        assert after["contacts"] == ref["contacts"]
        total += ref["contacts"]
        for k in ("vel", "ang", "rel", "pos", "pvel"):
            assert np.array_equal(after[k], ref[k]), k
    assert total > 500


def test_gather_and_solver_match_the_reference_host_loops(ctx):
    """ar_gather_contacts and ar_sequential_impulse against tests/golden/sis_solve.npz: the
    output of the reference's own GatherRigidBodyCollisions / GatherAugmentedRealityCollisions
    and SequentialImpulseSolver (Particles/updateFunctions.cpp:1431-1874) built for the host.
    Body-body contacts gathered and solved on the device; the reference's one-body (static
    scene) contacts solved on the device.  Bit for bit."""
    z = np.load(GOLDEN / "sis_solve.npz")
    n = len(z["rb_idx"])
    prm = api.sim_params(float(z["radius"]), (0, 0, 0), float(z["cell"]), z["dims"])
    prm.rb_restitution = float(z["restitution"])
    keys = ("normal", "point", "body1", "body2", "bias")
    out = {"normal": empty((n, 4)), "point": empty((n, 4)), "body1": empty(n, torch.int32),
           "body2": empty(n, torch.int32), "bias": empty(n), "acc0": empty(n), "acc1": empty(n),
           "acc2": empty(n)}
    cnt = empty(1, torch.int32)
    call("ar_gather_contacts", ctx.handle, C.byref(prm), n, P(dev(z["rb_idx"])), P(dev(z["cms"])),
         P(dev(z["vel"])), P(dev(z["ang"])), P(dev(z["rel"])), P(dev(z["contact_distance"])),
         P(dev(z["contact_body"])), P(dev(z["contact_particle"])), n, P(out["normal"]),
         P(out["point"]), P(out["body1"]), P(out["body2"]), P(out["bias"]), P(out["acc0"]),
         P(out["acc1"]), P(out["acc2"]), P(cnt), S())
    ctx.check()
    k = int(host(cnt)[0])
    assert k == len(z["rb_body1"]) > 1000
    gathered = {key: host(out[key])[:k] for key in keys}
    for key in keys:
        assert np.array_equal(gathered[key], z["rb_" + key]), key
    for tag, contacts in (("rb", gathered), ("ar", {key: z["ar_" + key] for key in keys})):
        v, w, acc = _solve_gpu(ctx, contacts, z["cms"], z["vel"], z["ang"], z["inv_inertia"],
                               z["mass"], int(z["iterations"]))
        assert np.array_equal(v, z[tag + "_vel"]) and np.array_equal(w, z[tag + "_ang"]), tag
        for i in range(3):
            assert np.array_equal(acc[i], z[tag + "_acc"][:, i]), (tag, i)
