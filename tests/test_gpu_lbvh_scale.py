"""LBVH at benchmark sizes: uniform points and a Gaussian mixture with 5 % exact duplicates,
30- and 63-bit Morton codes.  At 2^20 points the codes, the sort permutation and the tree
topology equal the oracle's bit for bit; at 2^24 points the size-independent properties are
checked on the device: keys non-decreasing with ties in index order, the permutation is a
permutation, every internal node's range is the union of its children's, parent links invert
child links, every node is reached once from the root, and every refitted box contains its
children's boxes."""
import numpy as np
import pytest
import torch

from diploma_thesis_b200 import scenes
from gpu_util import P, S, call, dev, empty, host
from oracle import cpu

pytestmark = pytest.mark.gpu


def _pipeline(ctx, pts: np.ndarray, wide: bool):
    n = len(pts)
    d = dev(pts)
    mn, mx = empty(4), empty(4)
    call("ar_scene_aabb", ctx.handle, P(d), n, P(mn), P(mx), S())
    kdt = torch.int64 if wide else torch.int32
    codes, skeys = empty(n, kdt), empty(n, kdt)
    svals = empty(n, torch.int32)
    call("ar_morton63" if wide else "ar_morton30", ctx.handle, P(d), n, P(mn), P(mx), P(codes),
         None, S())
    call("ar_radix_sort_pairs_u64" if wide else "ar_radix_sort_pairs_u32", ctx.handle, P(codes),
         None, P(skeys), P(svals), n, 0, 63 if wide else 30, S())
    m = 2 * n - 1
    t = {k: empty(m, torch.int32) for k in ("left", "right", "parent", "min_r", "max_r")}
    t["is_leaf"] = empty(m, torch.uint8)
    call("ar_lbvh_build64" if wide else "ar_lbvh_build", ctx.handle, P(skeys), n,
         P(t["is_leaf"]), P(t["left"]), P(t["right"]), P(t["parent"]), P(t["min_r"]),
         P(t["max_r"]), S())
    cms, bounds, radii = empty((n, 4)), empty((m, 8)), empty(n)
    call("ar_lbvh_leaves", ctx.handle, n, P(svals), P(d), 1e-3, P(t["is_leaf"]), P(t["min_r"]),
         P(t["max_r"]), P(cms), P(bounds), P(radii), S())
    call("ar_lbvh_refit", ctx.handle, n, P(t["left"]), P(t["right"]), P(t["parent"]),
         P(bounds), S())
    ctx.check()
    return d, mn, mx, codes, skeys, svals, t, bounds


@pytest.mark.parametrize("dist", ["uniform", "gmm"])
@pytest.mark.parametrize("wide", [False, True])
def test_lbvh_1m_bit_exact(ctx, dist, wide):
    n = 1 << 20
    pts = scenes.lbvh_points(n, dist, seed=3)
    d, mn, mx, codes, skeys, svals, t, bounds = _pipeline(ctx, pts, wide)
    mn4, mx4 = cpu.aabb(pts)
    assert np.array_equal(host(mn), mn4) and np.array_equal(host(mx), mx4)
    ref_codes = cpu.morton63(pts, mn4, mx4) if wide else cpu.morton30(pts, mn4, mx4)
    kt = np.uint64 if wide else np.uint32
    assert np.array_equal(host(codes, kt), ref_codes)
    k_ref, v_ref = cpu.sort_pairs(ref_codes, None, 0, 63 if wide else 30)
    assert np.array_equal(host(skeys, kt), k_ref)
    assert np.array_equal(host(svals, np.uint32), v_ref)
    if dist == "gmm":
        assert (k_ref[1:] == k_ref[:-1]).sum() > n // 40  # duplicates exercise the tie-break
    tr = cpu.radix_tree(k_ref)
    for k in ("left", "right", "min_r", "max_r"):
        assert np.array_equal(host(t[k])[n:], tr[k][n:]), k
    assert np.array_equal(host(t["parent"]), tr["parent"])  # root's parent -1 in both
    _, leaf_bounds = cpu.leaves(tr, v_ref, pts, 1e-3)
    ref_bounds = cpu.refit(tr, leaf_bounds)
    assert np.array_equal(host(bounds), ref_bounds)


def _device_tree_checks(n, skeys, svals, t, bounds):
    dev_ = skeys.device
    k = skeys
    # keys sorted, ties in index order, values a permutation
    assert bool((k[1:] >= k[:-1]).all())
    tie = k[1:] == k[:-1]
    assert bool((svals[1:][tie] > svals[:-1][tie]).all())
    seen = torch.zeros(n, dtype=torch.int32, device=dev_)
    seen.index_add_(0, svals.long(), torch.ones(n, dtype=torch.int32, device=dev_))
    assert bool((seen == 1).all())
    left, right, parent = t["left"].long(), t["right"].long(), t["parent"].long()
    min_r, max_r, leaf = t["min_r"].long(), t["max_r"].long(), t["is_leaf"]
    inner = torch.arange(n, 2 * n - 1, device=dev_)
    assert bool((leaf[:n] == 1).all()) and bool((leaf[n:] == 0).all())
    lc, rc = left[inner], right[inner]
    assert bool(((lc >= 0) & (lc < 2 * n - 1) & (rc >= 0) & (rc < 2 * n - 1)).all())
    assert bool((parent[lc] == inner).all()) and bool((parent[rc] == inner).all())
    assert bool((min_r[inner] == min_r[lc]).all()) and bool((max_r[inner] == max_r[rc]).all())
    assert bool((max_r[lc] + 1 == min_r[rc]).all())
    assert int(min_r[n]) == 0 and int(max_r[n]) == n - 1
    # every node except the root is exactly one node's child
    hits = torch.zeros(2 * n - 1, dtype=torch.int32, device=dev_)
    ones = torch.ones(n - 1, dtype=torch.int32, device=dev_)
    hits.index_add_(0, lc, ones)
    hits.index_add_(0, rc, ones)
    assert int(hits[n]) == 0
    hits[n] = 1
    assert bool((hits == 1).all())
    # refitted boxes contain their children's
    b = bounds
    for c in (lc, rc):
        assert bool((b[inner, :3] <= b[c, :3]).all()) and bool((b[inner, 3:6] >= b[c, 3:6]).all())


@pytest.mark.parametrize("dist,wide", [("uniform", False), ("gmm", True)])
def test_lbvh_16m_properties(ctx, dist, wide):
    n = 1 << 24
    pts = scenes.lbvh_points(n, dist, seed=4)
    d, mn, mx, codes, skeys, svals, t, bounds = _pipeline(ctx, pts, wide)
    del d, codes
    _device_tree_checks(n, skeys, svals, t, bounds)
