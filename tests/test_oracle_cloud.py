"""The oracle's fused step with a static point cloud (or_step_ex): no cloud and a cloud out of
reach give the plain step, and the cloud's impulse on each particle equals a float64 numpy
restatement of FindAndHandleAugmentedRealityCollisionsUniformGridKernel's law
(RigidBodies/UniformGridDEM.cu:243-377) summed over the points within 2r."""
import numpy as np

from diploma_thesis_b200 import scenes
from oracle import cpu

STATE = ("pos", "quat", "vel", "angvel")


def _cloud(seed, m, lo, hi):
    rng = np.random.default_rng(seed)
    pos = np.zeros((m, 4), np.float32)
    pos[:, :3] = rng.uniform(lo, hi, (m, 3))
    n = rng.normal(size=(m, 3))
    nrm = np.zeros((m, 4), np.float32)
    nrm[:, :3] = n / np.linalg.norm(n, axis=1, keepdims=True)
    return pos, nrm


def _rotate(q, v):
    """Rotate v by unit quaternions q = (x, y, z, w), float64."""
    u, w = q[:, :3], q[:, 3:4]
    t = 2.0 * np.cross(u, v)
    return v + w * t + np.cross(u, t)


def test_empty_and_far_clouds_give_the_plain_step():
    sc = scenes.small_scene(31, nb_side=3, r=1 / 128)
    plain = cpu.step(sc, 3)
    empty = cpu.step(sc, 3, cloud=(np.zeros((0, 4), np.float32), np.zeros((0, 4), np.float32)))
    far = cpu.step(sc, 3, cloud=_cloud(32, 500, 5.0, 6.0))  # wraps onto the grid, out of reach
    for k in STATE:
        assert np.array_equal(empty[k], plain[k]), k
        assert np.array_equal(far[k], plain[k]), k
    assert np.array_equal(far["pforce"], plain["pforce"])


def test_cloud_impulse_matches_fp64_law():
    sc = scenes.small_scene(33, nb_side=3, r=1 / 128)
    cp, cn = _cloud(34, 6000, 0.25, 0.75)
    with_cloud = cpu.step(sc, 1, cloud=(cp, cn))
    plain = cpu.step(sc, 1)
    got = (with_cloud["pforce"][:, :3].astype(np.float64) -
           plain["pforce"][:, :3].astype(np.float64))
    # particle positions and velocities at the start of the step, float64
    b = sc.body_index()
    rel = sc.particle_rel[:, :3].astype(np.float64)
    q = sc.body_quat.astype(np.float64)[b]
    r_w = _rotate(q, rel)
    p = sc.body_pos[b, :3].astype(np.float64) + r_w
    v = sc.body_vel[b, :3].astype(np.float64) + np.cross(sc.body_angvel[b, :3].astype(np.float64),
                                                          r_w)
    thr = 2.0 * sc.radius
    k, dmp, shr, att = sc.spring, sc.damping, sc.shear, sc.attraction
    want = np.zeros_like(got)
    ambiguous = np.zeros(len(p), bool)
    c3, n3 = cp[:, :3].astype(np.float64), cn[:, :3].astype(np.float64)
    for i in range(len(p)):
        rp = c3 - p[i]
        d = np.linalg.norm(rp, axis=1)
        ambiguous[i] = (np.abs(d - thr) < 1e-5 * thr).any()
        hit = d < thr
        if not hit.any():
            continue
        nrm = -n3[hit]
        rv = -v[i]
        tv = rv - (nrm @ rv)[:, None] * nrm
        f = (-k * (thr - d[hit]))[:, None] * nrm + dmp * rv + shr * tv + att * rp[hit]
        want[i] = f.sum(0)
    ok = ~ambiguous
    assert (np.abs(want[ok]).sum(1) > 0).sum() > 100
    scale = np.abs(want[ok]).max()
    assert np.abs(got[ok] - want[ok]).max() <= 1e-4 * scale
