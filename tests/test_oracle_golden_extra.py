"""Oracle vs the reference's own kernel bodies for the momentum integrator
(integrateRigidBody), the free-particle integrator (integrate_functor), the collideD
particle variant, and ReduceRigidBodyVariables' semantics."""
import numpy as np

from conftest import golden
from oracle import cpu


def test_integrate_momentum_bit_exact():
    g = golden("reference_extra")
    st = {k[len("mom_in_"):]: v for k, v in g.items() if k.startswith("mom_in_")}
    out = cpu.integrate_momentum(st, float(g["mom_dt"]), g["mom_radii"], g["mom_inv_mass"],
                                 [0, 0, 0], [1, 1, 1], [0, -0.5, 0], -0.5, 0.999)
    for k in st:
        assert np.array_equal(out[k], g[f"mom_out_{k}"]), k
    assert not np.array_equal(out["cms"], st["cms"])


def test_integrate_particles_bit_exact():
    g = golden("reference_extra")
    p, v = cpu.integrate_particles(g["fp_pos"], g["fp_vel"], g["fp_rb"], 0.01, [0, 0, 0],
                                   [1, 1, 1], [0, -0.5, 0], 0.999, -0.5, 1 / 64)
    assert np.array_equal(p, g["fp_pos_out"]) and np.array_equal(v, g["fp_vel_out"])
    free = g["fp_rb"] == -1
    assert not np.array_equal(p[free], g["fp_pos"][free])
    assert np.array_equal(p[~free], g["fp_pos"][~free])


def test_collide_particles_variant_bit_exact():
    g = golden("reference_extra")
    d = golden("dem_small")
    prm5 = list(d["prm"]) + [float(d["radius"])]
    pf, pt, nv = cpu.collide_grid_particles([0, 0, 0], float(d["cell"]), d["dims"], prm5,
                                            g["cd_rb"], d["spos"], d["svel"], d["rel"], d["sidx"],
                                            d["cell_start"], d["cell_end"])
    assert np.array_equal(pf, g["cd_pforce"]) and np.array_equal(pt, g["cd_ptorque"])
    assert np.array_equal(nv, g["cd_newvel"])
    assert (np.abs(g["cd_newvel"]).sum(1) > 0).sum() > 10  # free particles updated


def test_reduce_rigid_body_variables_adds_and_flags_nan():
    rng = np.random.default_rng(0)
    pf = rng.normal(0, 1, (300, 4)).astype(np.float32)
    pt = rng.normal(0, 1, (300, 4)).astype(np.float32)
    starts = np.array([0, 40, 100, 250], np.int32)
    counts = np.array([40, 50, 150, 50], np.int32)  # particles 90..99 belong to no rigid body
    bf0 = rng.normal(0, 1, (4, 4)).astype(np.float32)
    bt0 = np.zeros((4, 4), np.float32)
    bf, bt, ok = cpu.reduce_rigid_body_variables(pf, pt, starts, counts, bf0, bt0)
    assert ok
    for b in range(4):
        s = pf[starts[b]:starts[b] + counts[b], :3].astype(np.float64).sum(0)
        np.testing.assert_allclose(bf[b, :3], bf0[b, :3] + s, rtol=1e-5, atol=1e-5)
    pf[45, 1] = np.nan
    assert not cpu.reduce_rigid_body_variables(pf, pt, starts, counts, bf0, bt0)[2]


def test_static_scene_collisions_match_reference():
    """FindAndHandleAugmentedRealityCollisionsUniformGridKernel: particles against a static
    point cloud with normals (RigidBodies/UniformGridDEM.cu:243-377)."""
    g = golden("static_scene")
    c = float(g["cell"])
    lin, ang, color = cpu.collide_static_scene(
        (0.0, 0.0, 0.0), (c, c, c), g["dims"], float(g["radius"]), g["prm"], g["spos"],
        g["svel"], g["rel"], g["scene_spos"], g["scene_normals"], g["sidx"], g["scene_sidx"],
        g["scene_cell_start"], g["scene_cell_end"], g["lin0"], g["ang0"])
    assert (g["color"][:, 1] == 1).sum() > 100
    assert np.array_equal(lin, g["lin"]) and np.array_equal(ang, g["ang"])
    assert np.array_equal(color, g["color"])
