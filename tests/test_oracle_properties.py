"""Properties of the oracle that hold independently of the reference (CPU only), plus a CPU
check of the bit tricks the CUDA Morton encoder uses."""
import numpy as np
import pytest

from diploma_thesis_b200 import scenes
from oracle import cpu


def test_sort_is_stable_and_matches_numpy():
    rng = np.random.default_rng(0)
    for n, bits in [(0, 8), (1, 32), (777, 5), (10000, 21), (4096, 32)]:
        keys = rng.integers(0, 1 << bits, n, dtype=np.uint64).astype(np.uint32)
        k, v = cpu.sort_pairs(keys, None, 0, bits)
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(v, order) and np.array_equal(k, keys[order])


def test_sort_u64_begin_end_bits():
    rng = np.random.default_rng(1)
    keys = rng.integers(0, 1 << 63, 5000, dtype=np.uint64)
    k, v = cpu.sort_pairs(keys, None, 10, 40)
    digit = (keys >> np.uint64(10)) & np.uint64((1 << 30) - 1)
    assert np.array_equal(v, np.argsort(digit, kind="stable"))


def _spread10(v):  # the multiply-free shift/mask sequence the CUDA encoder uses
    v = v & 0x3FF
    v = (v | (v << 16)) & 0x030000FF
    v = (v | (v << 8)) & 0x0300F00F
    v = (v | (v << 4)) & 0x030C30C3
    v = (v | (v << 2)) & 0x09249249
    return v


def _spread21(v):
    v = v & 0x1FFFFF
    v = (v | (v << 32)) & 0x001F00000000FFFF
    v = (v | (v << 16)) & 0x001F0000FF0000FF
    v = (v | (v << 8)) & 0x100F00F00F00F00F
    v = (v | (v << 4)) & 0x10C30C30C30C30C3
    v = (v | (v << 2)) & 0x1249249249249249
    return v


def _naive(v, bits):
    out = 0
    for b in range(bits):
        out |= ((v >> b) & 1) << (3 * b)
    return out


def test_morton_spread_constants_exhaustive():
    for v in range(1024):
        assert _spread10(v) == _naive(v, 10)
        # the reference's multiply-and-mask expandBits (BVHSource/BVHkernels.cu:648-655)
        w = (v * 0x00010001) & 0xFF0000FF
        w = (w * 0x00000101) & 0x0F00F00F
        w = (w * 0x00000011) & 0xC30C30C3
        w = (w * 0x00000005) & 0x49249249
        assert w == _naive(v, 10)
    rng = np.random.default_rng(2)
    for v in list(rng.integers(0, 1 << 21, 3000)) + [0, 1, (1 << 21) - 1, 1 << 20]:
        assert _spread21(int(v)) == _naive(int(v), 21)


def test_morton_clamp_and_nan():
    pos = np.array([[-1, 0.5, 2, 0], [0.99999994, 1, 0, 0], [np.nan, 0.25, 0.5, 0],
                    [0.5, 0.5, 0.5, 0]], np.float32)
    mn = np.zeros(4, np.float32)
    mx = np.ones(4, np.float32)
    c = cpu.morton30(pos, mn, mx)
    assert c[1] == ((_spread10(1023) << 2) | (_spread10(1023) << 1))
    assert c[0] == ((_spread10(512) << 1) | _spread10(1023))
    assert c[2] == ((_spread10(256) << 1) | _spread10(512))  # NaN x clamps to 0
    c63 = cpu.morton63(pos, mn, mx)
    assert c63[3] == (_spread21(1 << 20) << 2) | (_spread21(1 << 20) << 1) | _spread21(1 << 20)


def _tree_is_valid(t, n):
    left, right, parent = t["left"], t["right"], t["parent"]
    lo, hi = t["min_r"], t["max_r"]
    seen = np.zeros(2 * n - 1, int)
    for node in range(n, 2 * n - 1):
        a, b = left[node], right[node]
        seen[a] += 1
        seen[b] += 1
        assert parent[a] == node and parent[b] == node
        assert lo[node] == lo[a] and hi[node] == hi[b] and hi[a] + 1 == lo[b]
    assert seen[n] == 0 and (seen[np.arange(2 * n - 1) != n] == 1).all()
    assert lo[n] == 0 and hi[n] == n - 1


@pytest.mark.parametrize("dup", [0.0, 0.3, 1.0])
def test_karras_topology_is_a_valid_binary_tree(dup):
    rng = np.random.default_rng(3)
    n = 4000
    codes = np.sort(rng.integers(0, 1 << 30, n).astype(np.uint32))
    if dup:
        m = int(n * dup)
        codes[:m] = codes[0] if dup == 1.0 else np.repeat(codes[: m // 4], 4)[:m]
        codes = np.sort(codes)
    t = cpu.radix_tree(codes)
    cpu.leaves(t, np.arange(n, dtype=np.int32), np.zeros((n, 4), np.float32), 0.0)
    _tree_is_valid(t, n)
    t64 = cpu.radix_tree(codes.astype(np.uint64) << np.uint64(30))
    for key in ("left", "right", "min_r", "max_r"):
        assert np.array_equal(t64[key][n:], t[key][n:])  # same order, same topology


def test_pair_sets_agree_across_broad_phases():
    """Brute force, grid (via the DEM gather's contact test) and BVH find the same pairs."""
    sc = scenes.small_scene(7, nb_side=5, packed=True)
    pos = sc.world_positions()
    rb = sc.body_index()
    two_r = np.float32(2 * sc.radius)
    brute = {tuple(p) for p in cpu.pairs_brute(pos, rb, two_r)}
    assert len(brute) > 200
    # BVH: contacts from the deepest-contact search are a subset; all contacts via DEM
    mn, mx = cpu.aabb(pos)
    k, v = cpu.sort_pairs(cpu.morton30(pos, mn, mx))
    t = cpu.radix_tree(k)
    cms, b = cpu.leaves(t, v.astype(np.int32), pos, float(sc.radius))
    b = cpu.refit(t, b)
    vel = np.zeros_like(pos)
    pf, _, _ = cpu.collide_bvh_dem([1.0, 0, 0, 0], rb, sc.particle_rel, vel, t, cms, b,
                                   v.astype(np.int32), np.full(len(pos), sc.radius, np.float32))
    touched = {i for p in brute for i in p}
    assert touched == set(np.flatnonzero(np.abs(pf).sum(1) > 0))


def test_physical_step_f32_tracks_f64():
    sc = scenes.small_scene(4, nb_side=3, packed=True, r=1 / 128)
    s32 = cpu.step(sc, steps=20)
    s64 = cpu.step_f64(sc, steps=20)
    assert s32["finite"] and s64["finite"]
    assert np.abs(s32["pos"][:, :3] - s64["pos"][:, :3]).max() < 1e-4 * sc.radius
