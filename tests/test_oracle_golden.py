"""The oracle (oracle/oracle.c) against golden vectors made by the reference's own kernel
bodies (tests/golden/make_golden.py).  Bit-exact everywhere except the per-body reduction,
where the reference's scan-difference with its one-element-late segment start
(RigidBodies/UniformGridDEM.cu:440-441) is a documented difference."""
import numpy as np
import pytest

from conftest import golden
from oracle import cpu, ref


@pytest.mark.parametrize("case", ["lbvh_uniform", "lbvh_duplicates"])
def test_lbvh_pipeline_bit_exact(case):
    g = golden(case)
    mn, mx = cpu.aabb(g["pos"])
    assert np.array_equal(mn, g["mn"]) and np.array_equal(mx, g["mx"])
    codes = cpu.morton30(g["pos"], mn, mx)
    assert np.array_equal(codes, g["codes"])
    k, v = cpu.sort_pairs(codes)
    assert np.array_equal(k, g["skeys"]) and np.array_equal(v, g["svals"])
    t = cpu.radix_tree(k)
    n = len(k)
    for key in ("left", "right", "min_r", "max_r", "is_leaf"):
        assert np.array_equal(t[key][n:], g[key][n:]), key
    # parent of every node but the root (the reference never writes the root's parent)
    par_ref = g["parent"].copy()
    par = t["parent"].copy()
    par_ref[n] = par[n] = -1
    assert np.array_equal(par, par_ref)
    cms, b = cpu.leaves(t, v.astype(np.int32), g["pos"], float(g["radius"]))
    assert np.array_equal(cms, g["cms"])
    assert np.array_equal(b[:n, :6], g["leaf_bounds"][:n, :6])
    b = cpu.refit(t, b)
    assert np.array_equal(b[:, :6], g["bounds"][:, :6])


def test_grid_dem_bit_exact():
    g = golden("dem_small")
    h = cpu.calc_hash([0, 0, 0], float(g["cell"]), g["dims"], g["pos"])
    assert np.array_equal(h, g["hash"])
    sh, si = cpu.sort_pairs(h)
    assert np.array_equal(sh, g["shash"]) and np.array_equal(si, g["sidx"])
    cs, ce, sp, sv = cpu.reorder(sh, si, g["pos"], g["vel"], int(np.prod(g["dims"])))
    occ = cs != 0xffffffff
    assert np.array_equal(cs, g["cell_start"])
    assert np.array_equal(ce[occ], g["cell_end"][occ])
    assert np.array_equal(sp, g["spos"]) and np.array_equal(sv, g["svel"])
    prm5 = list(g["prm"]) + [float(g["radius"])]
    pf, pt = cpu.collide_grid_dem([0, 0, 0], float(g["cell"]), g["dims"], prm5, g["rb"], sp, sv,
                                  g["rel"], si, cs, ce)
    assert np.array_equal(pf, g["pforce"])
    assert np.array_equal(pt, g["ptorque"])
    assert (np.abs(pf).sum(1) > 0).sum() > 100  # the case has contacts


def test_bvh_dem_and_contacts_bit_exact():
    g = golden("dem_small")
    t = cpu.radix_tree(g["bvh_keys"])
    idx = g["bvh_idx"].astype(np.int32)
    cms, _ = cpu.leaves(t, idx, g["pos"], float(g["radius"]))  # leaf flags come from here
    assert np.array_equal(cms, g["cms"])
    pf, pt, pp = cpu.collide_bvh_dem(g["prm"], g["rb"], g["rel"], g["vel"], t, g["cms"],
                                     g["bounds"], idx, g["radii"])
    assert np.array_equal(pf, g["bvh_pforce"])
    assert np.array_equal(pt, g["bvh_ptorque"])
    assert np.array_equal(pp, g["bvh_ppos"])
    cd, cp, cb = cpu.find_contacts_bvh(g["rb"], t, g["cms"], g["bounds"], idx, g["radii"],
                                       np.zeros(len(idx), np.float32))
    m = cd > 0
    assert m.sum() > 100
    assert np.array_equal(cd, g["contact_distance"])
    assert np.array_equal(cp[m], g["contact_particle"][m])
    assert np.array_equal(cb[m], g["contact_body"][m])


def test_grid_and_bvh_forces_agree():
    """Same contacts through both broad phases; only the summation order differs."""
    g = golden("dem_small")
    scale = np.abs(g["pforce"][:, :3]).max()
    assert np.abs(g["pforce"] - g["bvh_pforce"]).max() <= 1e-5 * scale


def test_reference_reduction_differs_only_by_its_segment_defect():
    """The fixed-order segmented sum against the reference's scan differences: the reference
    total of body b misses the body's first particle (its segment starts one element late)."""
    g = golden("dem_small")
    off = g["offsets"]
    v, a = cpu.reduce_impulses(g["pforce"], g["ptorque"], off, g["bvel"], g["bang"],
                               g["body_mass"], g["body_inv_inertia"])
    # emulate the defect: drop each body's first particle (except body 0), then compare
    pf, pt = g["pforce"].copy(), g["ptorque"].copy()
    pf[off[1:-1]] = 0
    pt[off[1:-1]] = 0
    v2, a2 = cpu.reduce_impulses(pf, pt, off, g["bvel"], g["bang"], g["body_mass"],
                                 g["body_inv_inertia"])
    scale_v = np.abs(g["ref_reduced_vel"]).max()
    # scan-difference cancellation leaves float32 noise relative to the running prefix
    assert np.abs(v2 - g["ref_reduced_vel"]).max() <= 2e-5 * max(scale_v, 1.0) * len(pf) ** 0.5
    assert not np.allclose(v, g["ref_reduced_vel"], atol=1e-6)


def test_body_stages_bit_exact():
    g = golden("bodies_small")
    st = {"cms": g["in_cms"], "vel": g["in_vel"], "ang": g["in_ang"], "quat": g["in_quat"],
          "ib": g["ib"], "cur": np.zeros_like(g["out_cur"]), "model": np.zeros_like(g["out_model"]),
          "cum": g["in_cum"]}
    out = cpu.integrate_reference(g["gravity"], float(g["w_damping"]), float(g["dt"]), st)
    # cos/sin come from the C library on both sides here, so the match is exact
    for k, gk in [("cms", "out_cms"), ("vel", "out_vel"), ("ang", "out_ang"), ("quat", "out_quat"),
                  ("cur", "out_cur"), ("model", "out_model"), ("cum", "out_cum")]:
        assert np.array_equal(out[k], g[gk]), k
    rel, pos, vel, q = cpu.global_attributes(g["out_cms"], g["out_vel"], g["out_ang"],
                                             g["out_quat"], g["rb"], g["in_rel"])
    assert np.array_equal(rel, g["out_rel"]) and np.array_equal(pos, g["out_pos"])
    assert np.array_equal(vel, g["out_pvel"]) and np.array_equal(q, g["out_q_reset"])
    v, a = cpu.walls_reference(float(g["radius"]), g["wall_ppos"], g["wall_bpos"], [0, 0, 0],
                               [1, 1, 1], g["wall_vel_in"], g["wall_ang_in"], g["ib"], g["mass"],
                               g["rb"], g["offsets"])
    assert np.array_equal(v, g["wall_vel_out"]) and np.array_equal(a, g["wall_ang_out"])
    assert not np.array_equal(v, g["wall_vel_in"])  # some bodies were hit


@pytest.mark.skipif(not ref.available(), reason="reference CPU build not present")
def test_live_reference_matches_oracle_on_fresh_inputs():
    """With the reference checkout built, check a fresh seeded case live (not only fixtures)."""
    rng = np.random.default_rng(123)
    pos = np.zeros((5000, 4), np.float32)
    pos[:, :3] = rng.random((5000, 3))
    pos[1::9] = pos[::9][: len(pos[1::9])]
    mn, mx = ref.aabb(pos)
    c_ref, idx = ref.morton30(pos, mn, mx)
    assert np.array_equal(cpu.morton30(pos, mn, mx), c_ref)
    k_ref, v_ref = ref.sort_pairs_u32(c_ref, idx.view(np.uint32))
    k, v = cpu.sort_pairs(c_ref)
    assert np.array_equal(k, k_ref) and np.array_equal(v, v_ref)
    t_ref, t = ref.radix_tree(k_ref), cpu.radix_tree(k)
    n = len(k)
    for key in ("left", "right", "min_r", "max_r"):
        assert np.array_equal(t[key][n:], t_ref[key][n:])
