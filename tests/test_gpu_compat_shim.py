"""The C++ shim (include/arsim_compat.hpp) run on the GPU through its reference signatures.

tests/compat_driver.cpp compiles the shim against the reference's own headers; here its
wrappers run on device buffers and are checked against the golden fixtures made by the
reference's own kernel bodies (tests/golden/make_golden.py):

* calcHash -> sortParticlesPreallocated -> reorderDataAndFindCellStart ->
  FindAndHandleRigidBodyCollisionsUniformGridWrapper on the dem_small scene: hashes, the
  stable permutation, cell ranges, sorted state and per-particle DEM forces / torques bit for
  bit, and the `**` swap (afterwards *hash and *index point at the sorted data, the sorted
  pointers at the spare buffers, as cub::DoubleBuffer::Current / Alternate);
* sortParticles: sorted in place, pointers unchanged, no device memory taken by a repeat call;
* ReducePerParticleImpulses with host-side counts: the oracle's fixed-order sums (the shim does
  not reproduce the reference's prefix-sum differences, which drop each body's first particle);
* WallCollisionWrapper: the reference's Baraff wall impulses bit for bit;
* loadRangeImage: the depth image's point cloud, vertex records and normals bit for bit.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import golden
from diploma_thesis_b200 import api
from gpu_util import dev, empty, host
from oracle import cpu

pytestmark = pytest.mark.gpu

try:
    from compat_build import LIB
except ImportError:  # pragma: no cover
    LIB = None


@pytest.fixture(scope="module")
def drv(ctx):
    if LIB is None or not LIB.exists():
        pytest.skip("tests/_compat/libcompat_driver.so not built (needs the reference headers)")
    d = C.CDLL(str(LIB))
    assert d.drv_sizeof_simparams() == C.sizeof(api.SimParams)
    assert d.drv_init() == 0
    return d


def _p(t: torch.Tensor) -> C.c_void_p:
    """Device pointer that keeps its tensor alive for as long as the pointer object (temporary
    tensors passed to a call must not be freed before the call returns)."""
    return api.ptr(t)


def _params(g) -> api.SimParams:
    return api.sim_params(float(g["radius"]), (0, 0, 0), float(g["cell"]), g["dims"],
                          *[float(x) for x in g["prm"]])


def test_grid_path_through_the_shim_golden(drv):
    g = golden("dem_small")
    n = len(g["pos"])
    ncell = int(np.prod(g["dims"]))
    prm = _params(g)
    drv.drv_set_params(C.byref(prm))
    pos, vel = dev(g["pos"]), dev(g["vel"])
    h, idx = empty(n, torch.int32), empty(n, torch.int32)
    drv.drv_calc_hash(_p(h), _p(idx), _p(pos), n)
    assert drv.drv_take_status() == 0
    assert np.array_equal(host(h, np.uint32), g["hash"])
    sh, si = empty(n, torch.int32), empty(n, torch.int32)
    out = (C.c_void_p * 4)()
    drv.drv_sort_preallocated(_p(h), _p(idx), _p(sh), _p(si), n, out)
    assert drv.drv_take_status() == 0
    # the `**` swap: *hash / *index now name the sorted buffers, the sorted pointers the spares
    assert [out[i] for i in range(4)] == [sh.data_ptr(), si.data_ptr(), h.data_ptr(), idx.data_ptr()]
    assert np.array_equal(host(sh, np.uint32), g["shash"])
    assert np.array_equal(host(si, np.uint32), g["sidx"])
    cs, ce = empty(ncell, torch.int32), empty(ncell, torch.int32)
    sp, sv = empty((n, 4)), empty((n, 4))
    drv.drv_reorder(_p(cs), _p(ce), _p(sp), _p(sv), _p(sh), _p(si), _p(pos), _p(vel), n, ncell)
    assert drv.drv_take_status() == 0
    occ = g["cell_start"] != 0xffffffff
    assert np.array_equal(host(cs, np.uint32), g["cell_start"])
    assert np.array_equal(host(ce, np.uint32)[occ], g["cell_end"][occ])
    assert np.array_equal(host(sp), g["spos"]) and np.array_equal(host(sv), g["svel"])
    pf, pt = empty((n, 4)), empty((n, 4))
    drv.drv_collide_grid_dem(C.byref(prm), _p(dev(g["rb"])), _p(pf), _p(pt), _p(sp), _p(sv),
                             _p(dev(g["rel"])), _p(si), _p(cs), _p(ce), n)
    assert drv.drv_take_status() == 0
    assert np.array_equal(host(pf), g["pforce"]) and np.array_equal(host(pt), g["ptorque"])


def test_sort_in_place_through_the_shim(drv):
    rng = np.random.default_rng(5)
    for n in (1000, 300_001, 1000):  # grow, then a repeat call that reuses the spare buffers
        keys = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
        keys[: n // 3] = keys[n // 3: 2 * (n // 3)]
        vals = rng.integers(0, 1 << 31, n).astype(np.uint32)
        k, v = dev(keys), dev(vals)
        out = (C.c_void_p * 2)()
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        drv.drv_sort_in_place(_p(k), _p(v), n, out)
        assert drv.drv_take_status() == 0
        assert [out[0], out[1]] == [k.data_ptr(), v.data_ptr()]  # in place: pointers unchanged
        k_ref, v_ref = cpu.sort_pairs(keys, vals, 0, 32)
        assert np.array_equal(host(k, np.uint32), k_ref)
        assert np.array_equal(host(v, np.uint32), v_ref)
        if n == 1000:  # smaller than an earlier call: nothing allocated
            assert torch.cuda.mem_get_info()[0] == free_before


def test_reduce_impulses_through_the_shim(drv):
    g = golden("dem_small")
    off = g["offsets"]
    nb = len(off) - 1
    n = int(off[-1])
    counts = np.ascontiguousarray(np.diff(off).astype(np.int32))
    vel, ang = dev(g["bvel"]), dev(g["bang"])
    drv.drv_reduce_impulses(_p(dev(g["rb"])), _p(dev(g["pforce"])), _p(dev(g["ptorque"])),
                            _p(vel), _p(ang), _p(dev(g["body_mass"])),
                            _p(dev(g["body_inv_inertia"])),
                            counts.ctypes.data_as(C.POINTER(C.c_int)), nb, n)
    assert drv.drv_take_status() == 0
    v_ref, a_ref = cpu.reduce_impulses(g["pforce"], g["ptorque"], off, g["bvel"], g["bang"],
                                       g["body_mass"], g["body_inv_inertia"])
    assert np.array_equal(host(vel), v_ref) and np.array_equal(host(ang), a_ref)


def test_walls_through_the_shim(drv):
    g = golden("bodies_small")
    nb = len(g["wall_bpos"])
    n = len(g["wall_ppos"])
    prm = api.sim_params(float(g["radius"]), (0, 0, 0), 1.0, (1, 1, 1))
    counts = np.ascontiguousarray(np.diff(g["offsets"]).astype(np.int32))
    vel, ang = dev(g["wall_vel_in"]), dev(g["wall_ang_in"])
    mn = (C.c_float * 3)(0, 0, 0)
    mx = (C.c_float * 3)(1, 1, 1)
    drv.drv_walls(C.byref(prm), _p(dev(g["wall_ppos"])), _p(dev(g["wall_bpos"])), mn, mx,
                  _p(vel), _p(ang), _p(dev(g["ib"])), _p(dev(g["mass"])), _p(dev(g["rb"])),
                  counts.ctypes.data_as(C.POINTER(C.c_int)), nb, n)
    assert drv.drv_take_status() == 0
    assert np.array_equal(host(vel), g["wall_vel_out"])
    assert np.array_equal(host(ang), g["wall_ang_out"])


def test_load_range_image_through_the_shim(drv):
    # loadRangeImage(image, &VAOdata, &staticPos, &staticNorm, camera, radii, r, w, h): the
    # reference's cloud, vertex records and normals bit for bit
    z = golden("range_image")
    h, w = z["depth"].shape
    depth = torch.from_numpy(z["depth"].view(np.int16).copy()).cuda()
    bufs = {k: torch.full(shape, float("nan"), device="cuda") for k, shape in
            (("vao5", (h * w, 5)), ("pos4", (h * w, 4)), ("norm4", (h * w, 4)),
             ("radii", (h * w,)))}
    cam = np.ascontiguousarray(z["camera16"].astype(np.float32))
    rc = drv.drv_range_image(_p(depth), _p(bufs["vao5"]), _p(bufs["pos4"]), _p(bufs["norm4"]),
                             _p(bufs["radii"]), cam.ctypes.data_as(C.c_void_p),
                             C.c_float(float(z["radius"])), w, h)
    assert rc == 0 and drv.drv_take_status() == 0
    for k, t in bufs.items():
        got, want = host(t), z[k]
        written = ~np.isnan(want)
        assert np.array_equal(~np.isnan(got), written)
        assert np.array_equal(got[written].view(np.uint32), want[written].view(np.uint32)), k
