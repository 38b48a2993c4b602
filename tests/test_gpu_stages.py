"""Each CUDA stage entry point, called through the C ABI, against the golden fixtures made by
the reference's own kernel bodies and against the oracle.  Integer / index outputs must be
bit-exact; float outputs are bit-exact where the arithmetic is + - * / sqrt (the library is
built without FMA contraction), and within 1e-5 relative where the reference uses cos/sin."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import golden
from diploma_thesis_b200 import api, scenes
from gpu_util import F3, F4, P, S, call, dev, empty, host
from oracle import cpu

pytestmark = pytest.mark.gpu


# ---- (a6)/(a7) AABB and Morton codes -----------------------------------------------------
@pytest.mark.parametrize("case", ["lbvh_uniform", "lbvh_duplicates"])
def test_aabb_morton30_golden(ctx, case):
    g = golden(case)
    n = len(g["pos"])
    pos = dev(g["pos"])
    mn, mx = empty(4), empty(4)
    call("ar_scene_aabb", ctx.handle, P(pos), n, P(mn), P(mx), S())
    assert np.array_equal(host(mn), g["mn"]) and np.array_equal(host(mx), g["mx"])
    codes, idx = empty(n, torch.int32), empty(n, torch.int32)
    call("ar_morton30", ctx.handle, P(pos), n, P(mn), P(mx), P(codes), P(idx), S())
    assert np.array_equal(host(codes, np.uint32), g["codes"])
    assert np.array_equal(host(idx), np.arange(n))
    codes2 = empty(n, torch.int32)
    call("ar_morton30_box", ctx.handle, P(pos), n, F4(*g["mn"]), F4(*g["mx"]), P(codes2), None, S())
    assert np.array_equal(host(codes2, np.uint32), g["codes"])


@pytest.mark.parametrize("n", [1, 2, 1000, 300001])
def test_morton_random_with_edges(ctx, n):
    rng = np.random.default_rng(n)
    pos = np.zeros((n, 4), np.float32)
    pos[:, :3] = rng.normal(0.5, 0.3, (n, 3))
    pos[: n // 10] = pos[n // 10: 2 * (n // 10)]  # duplicates
    if n > 10:
        pos[3, 0] = np.nan
        pos[4, 1] = 1e30
    mn4 = np.array([0, 0, 0, 0], np.float32)
    mx4 = np.array([1, 1, 1, 1], np.float32)
    d = dev(pos)
    c30, c63 = empty(n, torch.int32), empty(n, torch.int64)
    dmn, dmx = dev(mn4), dev(mx4)
    call("ar_morton30", ctx.handle, P(d), n, P(dmn), P(dmx), P(c30), None, S())
    call("ar_morton63", ctx.handle, P(d), n, P(dmn), P(dmx), P(c63), None, S())
    assert np.array_equal(host(c30, np.uint32), cpu.morton30(pos, mn4, mx4))
    assert np.array_equal(host(c63, np.uint64), cpu.morton63(pos, mn4, mx4))


# ---- (a8) radix sort --------------------------------------------------------------------------
@pytest.mark.parametrize("n,bits", [(1, 32), (2, 1), (4095, 8), (4096, 9), (4097, 16),
                                    (100003, 21), (1 << 20, 32), (777777, 30),
                                    # plans with 9-bit passes: 8+9; 8+9+9 with 256- and
                                    # 512-thread tiles in one sort; 8+8+9 at 2M keys
                                    (50001, 17), (300001, 26), ((1 << 21) + 3, 25)])
def test_sort_u32_matches_stable_order(ctx, n, bits):
    rng = np.random.default_rng(bits * 7 + n)
    keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32)
    keys[: n // 3] = keys[n // 3: 2 * (n // 3)]  # many ties
    vals = rng.integers(0, 1 << 31, n).astype(np.uint32)
    kin, vin = dev(keys), dev(vals)
    kout, vout = empty(n, torch.int32), empty(n, torch.int32)
    for use_vals in (False, True):
        call("ar_radix_sort_pairs_u32", ctx.handle, P(kin), P(vin) if use_vals else None,
             P(kout), P(vout), n, 0, bits, S())
        ctx.check()
        k_ref, v_ref = cpu.sort_pairs(keys, vals if use_vals else None, 0, bits)
        assert np.array_equal(host(kout, np.uint32), k_ref)
        assert np.array_equal(host(vout, np.uint32), v_ref)
    assert np.array_equal(host(kin, np.uint32), keys)  # inputs intact


def test_sort_u32_all_equal_and_begin_bit(ctx):
    n = 50000
    keys = np.full(n, 0xdeadbeef, np.uint32)
    kin = dev(keys)
    kout, vout = empty(n, torch.int32), empty(n, torch.int32)
    call("ar_radix_sort_pairs_u32", ctx.handle, P(kin), None, P(kout), P(vout), n, 0, 32, S())
    assert np.array_equal(host(vout), np.arange(n))
    rng = np.random.default_rng(9)
    keys = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    kin = dev(keys)
    call("ar_radix_sort_pairs_u32", ctx.handle, P(kin), None, P(kout), P(vout), n, 12, 28, S())
    assert np.array_equal(host(vout, np.uint32), cpu.sort_pairs(keys, None, 12, 28)[1])


@pytest.mark.parametrize("n,begin,end", [(5000, 0, 63), (100000, 3, 48), (4096, 0, 64)])
def test_sort_u64(ctx, n, begin, end):
    rng = np.random.default_rng(n)
    keys = rng.integers(0, 1 << 63, n, dtype=np.uint64)
    m = len(keys[1::5])
    keys[::5][:m] = keys[1::5]  # ties
    kin = dev(keys)
    kout, vout = empty(n, torch.int64), empty(n, torch.int32)
    call("ar_radix_sort_pairs_u64", ctx.handle, P(kin), None, P(kout), P(vout), n, begin, end, S())
    k_ref, v_ref = cpu.sort_pairs(keys, None, begin, end)
    assert np.array_equal(host(vout, np.uint32), v_ref)
    assert np.array_equal(host(kout, np.uint64), k_ref)


def test_sort_rejects_bad_arguments(ctx):
    from diploma_thesis_b200 import _lib
    k = empty(10, torch.int32)
    L = _lib.lib
    assert L.ar_radix_sort_pairs_u32(ctx.handle, P(k), None, P(k), P(k), 10, 0, 32, S()) == 1
    assert L.ar_radix_sort_pairs_u32(ctx.handle, P(k), None, P(empty(10, torch.int32)),
                                     P(empty(10, torch.int32)), 10, 0, 33, S()) == 1
    assert L.ar_radix_sort_pairs_u32(ctx.handle, None, None, None, None, 0, 0, 32, S()) == 0


# ---- (a9)-(a11) LBVH ---------------------------------------------------------------------------
def build_tree_gpu(ctx, skeys: np.ndarray, wide: bool = False):
    n = len(skeys)
    m = 2 * n - 1
    t = {k: empty(m, torch.int32) for k in ("left", "right", "parent", "min_r", "max_r")}
    t["is_leaf"] = empty(m, torch.uint8)
    kd = dev(skeys)
    name = "ar_lbvh_build64" if wide else "ar_lbvh_build"
    call(name, ctx.handle, P(kd), n, P(t["is_leaf"]), P(t["left"]), P(t["right"]),
         P(t["parent"]), P(t["min_r"]), P(t["max_r"]), S())
    return t


@pytest.mark.parametrize("case", ["lbvh_uniform", "lbvh_duplicates"])
def test_lbvh_topology_leaves_refit_golden(ctx, case):
    g = golden(case)
    n = len(g["skeys"])
    t = build_tree_gpu(ctx, g["skeys"])
    for key in ("left", "right", "min_r", "max_r"):
        assert np.array_equal(host(t[key])[n:], g[key][n:]), key
    par = host(t["parent"])
    par_ref = g["parent"].copy()
    assert par[n] == -1
    par_ref[n] = -1
    assert np.array_equal(par, par_ref)
    pos = dev(g["pos"])
    sidx = dev(g["svals"].astype(np.int32))
    cms, bounds, radii = empty((n, 4)), empty((2 * n - 1, 8)), empty(n)
    call("ar_lbvh_leaves", ctx.handle, n, P(sidx), P(pos), C.c_float(g["radius"]),
         P(t["is_leaf"]), P(t["min_r"]), P(t["max_r"]), P(cms), P(bounds), P(radii), S())
    assert np.array_equal(host(cms), g["cms"])
    assert np.array_equal(host(bounds)[:n, :6], g["leaf_bounds"][:n, :6])
    call("ar_lbvh_refit", ctx.handle, n, P(t["left"]), P(t["right"]), P(t["parent"]),
         P(bounds), S())
    assert np.array_equal(host(bounds)[:, :6], g["bounds"][:, :6])
    assert np.array_equal(host(t["is_leaf"]), np.r_[np.ones(n), np.zeros(n - 1)].astype(np.uint8))


@pytest.mark.parametrize("n,dup", [(2, 0.0), (3, 1.0), (1000, 0.5), (65537, 0.05)])
def test_lbvh_random_32_and_64(ctx, n, dup):
    rng = np.random.default_rng(n)
    c = np.sort(rng.integers(0, 1 << 30, n).astype(np.uint32))
    m = int(n * dup)
    if m:
        c[:m] = c[0]
        c = np.sort(c)
    ref = cpu.radix_tree(c)
    t = build_tree_gpu(ctx, c)
    for key in ("left", "right", "min_r", "max_r"):
        assert np.array_equal(host(t[key])[n:], ref[key][n:]), key
    c64 = (c.astype(np.uint64) << np.uint64(33)) | rng.integers(0, 2, n).astype(np.uint64)
    c64 = np.sort(c64)
    ref64 = cpu.radix_tree(c64)
    t64 = build_tree_gpu(ctx, c64, wide=True)
    for key in ("left", "right", "min_r", "max_r"):
        assert np.array_equal(host(t64[key])[n:], ref64[key][n:]), key


def _golden_tree_on_gpu(ctx, g):
    n = len(g["bvh_keys"])
    t = build_tree_gpu(ctx, g["bvh_keys"])
    sidx = dev(g["bvh_idx"].astype(np.int32))
    cms, bounds, radii = empty((n, 4)), empty((2 * n - 1, 8)), empty(n)
    call("ar_lbvh_leaves", ctx.handle, n, P(sidx), P(dev(g["pos"])), C.c_float(g["radius"]),
         P(t["is_leaf"]), P(t["min_r"]), P(t["max_r"]), P(cms), P(bounds), P(radii), S())
    call("ar_lbvh_refit", ctx.handle, n, P(t["left"]), P(t["right"]), P(t["parent"]),
         P(bounds), S())
    return t, sidx, cms, bounds, radii


def test_collide_bvh_dem_and_contacts_golden(ctx):
    g = golden("dem_small")
    n = len(g["pos"])
    t, sidx, cms, bounds, radii = _golden_tree_on_gpu(ctx, g)
    assert np.array_equal(host(bounds)[:, :6], g["bounds"][:, :6])
    prm = api.sim_params(float(g["radius"]), (0, 0, 0), float(g["cell"]), g["dims"],
                         *[float(x) for x in g["prm"]])
    pf, pt, pp = empty((n, 4)), empty((n, 4)), empty((n, 4))
    call("ar_collide_bvh_dem", ctx.handle, C.byref(prm), P(dev(g["rb"])), P(dev(g["rel"])),
         P(dev(g["vel"])), P(t["is_leaf"]), P(t["left"]), P(t["right"]), P(t["parent"]),
         P(cms), P(bounds), P(sidx), P(radii), n, P(pf), P(pt), P(pp), S())
    assert np.array_equal(host(pf), g["bvh_pforce"])
    assert np.array_equal(host(pt), g["bvh_ptorque"])
    assert np.array_equal(host(pp), g["bvh_ppos"])
    cd = empty(n)
    cp, cb = empty(n, torch.int32), empty(n, torch.int32)
    call("ar_find_contacts_bvh", ctx.handle, P(dev(g["rb"])), P(t["is_leaf"]), P(t["left"]),
         P(t["right"]), P(t["parent"]), P(t["max_r"]), P(cms), P(bounds), P(sidx), P(radii), n,
         P(cd), P(cp), P(cb), S())
    m = g["contact_distance"] > 0
    assert np.array_equal(host(cd), g["contact_distance"])
    assert np.array_equal(host(cp)[m], g["contact_particle"][m])
    assert np.array_equal(host(cb)[m], g["contact_body"][m])


def _pairs(ctx, fn_name, args, cap):
    pairs = empty((cap, 2), torch.int32)
    cnt = empty(1, torch.int32)
    call(fn_name, ctx.handle, *args, P(pairs), cap, P(cnt), S())
    ctx.check()
    k = int(host(cnt)[0])
    p = host(pairs)[:k]
    return {tuple(x) for x in p}, k


def test_pair_sets_grid_bvh_bruteforce_equal(ctx):
    g = golden("dem_small")
    n = len(g["pos"])
    brute = {tuple(x) for x in cpu.pairs_brute(g["pos"], g["rb"], np.float32(2 * g["radius"]))}
    t, sidx, cms, bounds, radii = _golden_tree_on_gpu(ctx, g)
    bvh, kb = _pairs(ctx, "ar_pairs_bvh", [C.c_float(g["radius"]), P(dev(g["rb"])), P(t["is_leaf"]),
                                            P(t["left"]), P(t["right"]), P(t["parent"]), P(cms),
                                            P(bounds), P(sidx), n], 200000)
    prm = api.sim_params(float(g["radius"]), (0, 0, 0), float(g["cell"]), g["dims"])
    grid, kg = _pairs(ctx, "ar_pairs_grid", [C.byref(prm), P(dev(g["rb"])), P(dev(g["spos"])),
                                              P(dev(g["sidx"])), P(dev(g["cell_start"])),
                                              P(dev(g["cell_end"])), n], 200000)
    assert len(brute) > 500
    assert bvh == brute and kb == len(brute)
    assert grid == brute and kg == len(brute)


def test_pair_overflow_reports_status(ctx):
    from diploma_thesis_b200 import _lib
    g = golden("dem_small")
    n = len(g["pos"])
    prm = api.sim_params(float(g["radius"]), (0, 0, 0), float(g["cell"]), g["dims"])
    pairs = empty((10, 2), torch.int32)
    cnt = empty(1, torch.int32)
    call("ar_pairs_grid", ctx.handle, C.byref(prm), P(dev(g["rb"])), P(dev(g["spos"])),
         P(dev(g["sidx"])), P(dev(g["cell_start"])), P(dev(g["cell_end"])), n, P(pairs), 10,
         P(cnt), S())
    assert ctx.status() == 7  # AR_ERR_OVERFLOW
    assert ctx.status() == 0  # cleared
    assert int(host(cnt)[0]) > 10


# ---- (a13)-(a15) grid path -------------------------------------------------------------------
def test_grid_hash_reorder_collide_golden(ctx):
    g = golden("dem_small")
    n = len(g["pos"])
    ncell = int(np.prod(g["dims"]))
    prm = api.sim_params(float(g["radius"]), (0, 0, 0), float(g["cell"]), g["dims"],
                         *[float(x) for x in g["prm"]])
    pos, vel = dev(g["pos"]), dev(g["vel"])
    h, idx = empty(n, torch.int32), empty(n, torch.int32)
    call("ar_calc_hash", ctx.handle, C.byref(prm), P(pos), n, P(h), P(idx), S())
    assert np.array_equal(host(h, np.uint32), g["hash"])
    sh, si = empty(n, torch.int32), empty(n, torch.int32)
    call("ar_radix_sort_pairs_u32", ctx.handle, P(h), P(idx), P(sh), P(si), n, 0, 32, S())
    assert np.array_equal(host(si, np.uint32), g["sidx"])
    cs, ce = empty(ncell, torch.int32), empty(ncell, torch.int32)
    sp, sv = empty((n, 4)), empty((n, 4))
    call("ar_reorder_cells", ctx.handle, P(sh), P(si), P(pos), P(vel), n, ncell, P(cs), P(ce),
         P(sp), P(sv), S())
    cs_h, ce_h = host(cs, np.uint32), host(ce, np.uint32)
    occ = g["cell_start"] != 0xffffffff
    assert np.array_equal(cs_h, g["cell_start"])
    assert np.array_equal(ce_h[occ], g["cell_end"][occ])
    assert np.array_equal(host(sp), g["spos"]) and np.array_equal(host(sv), g["svel"])
    pf, pt = empty((n, 4)), empty((n, 4))
    call("ar_collide_grid_dem", ctx.handle, C.byref(prm), P(dev(g["rb"])), P(sp), P(sv),
         P(dev(g["rel"])), P(si), P(cs), P(ce), n, P(pf), P(pt), S())
    assert np.array_equal(host(pf), g["pforce"])
    assert np.array_equal(host(pt), g["ptorque"])


def test_grid_rejects_non_power_of_two(ctx):
    from diploma_thesis_b200 import _lib
    prm = api.sim_params(0.01, (0, 0, 0), 0.02, (12, 16, 16))
    pos = empty((4, 4))
    h = empty(4, torch.int32)
    assert _lib.lib.ar_calc_hash(ctx.handle, C.byref(prm), P(pos), 4, P(h), None, S()) == 1


# ---- (a16)-(a18) per-body stages --------------------------------------------------------------
def test_reduce_bodies_bit_exact_and_impulses(ctx):
    g = golden("dem_small")
    off = g["offsets"]
    nb = len(off) - 1
    bf, bt = empty((nb, 4)), empty((nb, 4))
    call("ar_reduce_bodies", ctx.handle, P(dev(g["pforce"])), P(dev(g["ptorque"])), P(dev(off)),
         nb, P(bf), P(bt), S())
    rf, rt = cpu.reduce_bodies(g["pforce"], g["ptorque"], off)
    assert np.array_equal(host(bf), rf) and np.array_equal(host(bt), rt)
    vel, ang = dev(g["bvel"]), dev(g["bang"])
    call("ar_reduce_impulses", ctx.handle, P(dev(g["pforce"])), P(dev(g["ptorque"])), P(dev(off)),
         nb, P(vel), P(ang), P(dev(g["body_mass"])), P(dev(g["body_inv_inertia"])), S())
    v_ref, a_ref = cpu.reduce_impulses(g["pforce"], g["ptorque"], off, g["bvel"], g["bang"],
                                       g["body_mass"], g["body_inv_inertia"])
    assert np.array_equal(host(vel), v_ref) and np.array_equal(host(ang), a_ref)
    # against an FP64 segmented sum: within 1e-5 of the summed magnitudes
    f64 = np.array([g["pforce"][off[b]:off[b + 1], :3].astype(np.float64).sum(0) for b in range(nb)])
    mag = np.array([np.abs(g["pforce"][off[b]:off[b + 1], :3]).astype(np.float64).sum(0) for b in range(nb)])
    assert (np.abs(host(bf)[:, :3] - f64) <= 1e-5 * mag + 1e-12).all()


def test_reference_integrator_and_reposing_golden(ctx):
    g = golden("bodies_small")
    nb = len(g["in_cms"])
    cms, vel, ang, quat = (dev(g[k]) for k in ("in_cms", "in_vel", "in_ang", "in_quat"))
    cur, model, cum = empty((nb, 9)), empty((nb, 16)), dev(g["in_cum"])
    prm = api.sim_params(0.01, (0, 0, 0), 1.0, (1, 1, 1), gravity=tuple(g["gravity"]),
                         w_damping=float(g["w_damping"]))
    call("ar_integrate_reference", ctx.handle, C.byref(prm), C.c_float(g["dt"]), nb, P(cms),
         P(vel), P(ang), P(quat), P(dev(g["ib"])), P(cur), P(model), P(cum), P(dev(g["mass"])), S())
    # cos/sin differ between the CUDA and C libraries by an ulp at most
    for t, k in [(cms, "out_cms"), (vel, "out_vel"), (ang, "out_ang")]:
        assert np.array_equal(host(t), g[k]), k
    for t, k in [(quat, "out_quat"), (cur, "out_cur"), (model, "out_model"), (cum, "out_cum")]:
        np.testing.assert_allclose(host(t), g[k], rtol=1e-5, atol=1e-6, err_msg=k)
    # re-posing on the golden body state: bit-exact
    n = len(g["in_rel"])
    q = dev(g["out_quat"])
    rel, pos, pvel = dev(g["in_rel"]), empty((n, 4)), empty((n, 4))
    call("ar_global_attributes", ctx.handle, n, nb, P(dev(g["out_cms"])), P(dev(g["out_vel"])),
         P(dev(g["out_ang"])), P(q), P(dev(g["rb"])), P(rel), P(pos), P(pvel), S())
    assert np.array_equal(host(q), g["out_quat"])  # untouched until the reset
    call("ar_reset_quaternions", ctx.handle, P(q), nb, S())
    assert np.array_equal(host(rel), g["out_rel"]) and np.array_equal(host(pos), g["out_pos"])
    assert np.array_equal(host(pvel), g["out_pvel"]) and np.array_equal(host(q), g["out_q_reset"])


def test_reference_walls_golden(ctx):
    g = golden("bodies_small")
    nb = len(g["wall_bpos"])
    n = len(g["wall_ppos"])
    vel, ang = dev(g["wall_vel_in"]), dev(g["wall_ang_in"])
    call("ar_walls_reference", ctx.handle, C.c_float(g["radius"]), P(dev(g["wall_ppos"])),
         P(dev(g["wall_bpos"])), F3(0, 0, 0), F3(1, 1, 1), P(vel), P(ang), P(dev(g["ib"])),
         P(dev(g["mass"])), P(dev(g["rb"])), P(dev(g["offsets"])), nb, n, S())
    assert np.array_equal(host(vel), g["wall_vel_out"])
    assert np.array_equal(host(ang), g["wall_ang_out"])
