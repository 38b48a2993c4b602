"""numpy wrappers over oracle/_ref/libref_cpu.so -- the reference's own kernel bodies run on
the CPU (built from the reference checkout by oracle/ref_build.py).

TEST INFRASTRUCTURE ONLY.  Used to generate the golden fixtures, to pin oracle.cpu, and as
the CPU baseline of bench.py's reference arm.  ``available()`` is False where the library
was not built (no reference checkout when it was built).
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

_SO = Path(__file__).resolve().parent / "_ref" / "libref_cpu.so"
_L = None


class SimParams(C.Structure):
    """The reference's `struct SimParams` (Kernels/particleSystem.cuh:27-55), 128 bytes, as the
    reference build's kernels read it.  Declared here so that nothing on the reference's side
    (the golden-fixture generator, bench.py's reference arm) loads the product library."""
    _fields_ = [("collider_pos", C.c_float * 3), ("collider_radius", C.c_float),
                ("gravity", C.c_float * 3), ("global_damping", C.c_float),
                ("particle_radius", C.c_float), ("grid_size", C.c_uint32 * 3),
                ("num_cells", C.c_uint32), ("world_origin", C.c_float * 3),
                ("cell_size", C.c_float * 3), ("num_bodies", C.c_uint32),
                ("max_particles_per_cell", C.c_uint32), ("spring", C.c_float),
                ("damping", C.c_float), ("shear", C.c_float), ("attraction", C.c_float),
                ("boundary_damping", C.c_float), ("ar_restitution", C.c_float),
                ("rb_restitution", C.c_float), ("ar_friction", C.c_float),
                ("rb_friction", C.c_float), ("w_damping", C.c_float), ("v_damping", C.c_float)]


def sim_params(radius: float, grid_origin, cell, grid_dims, spring=0.5, damping=0.02,
               shear=0.1, attraction=0.0, gravity=(0.0, -9.81, 0.0), w_damping=1.0) -> SimParams:
    """Parameters as the reference's ParticleSystem sets them (Particles/particleSystem.cpp:
    123-141): global damping 1, boundary damping -0.5, the given grid and DEM constants."""
    p = SimParams()
    p.particle_radius = radius
    for a in range(3):
        p.world_origin[a] = grid_origin[a]
        p.cell_size[a] = cell[a] if np.ndim(cell) else cell
        p.grid_size[a] = int(grid_dims[a])
        p.gravity[a] = gravity[a]
    p.num_cells = int(np.prod(grid_dims))
    p.spring, p.damping, p.shear, p.attraction = spring, damping, shear, attraction
    p.w_damping = w_damping
    p.global_damping = 1.0
    p.boundary_damping = -0.5
    return p


def available() -> bool:
    return _SO.exists()


def lib():
    global _L
    if _L is None:
        if not _SO.exists():
            raise FileNotFoundError(f"{_SO} not built (needs the reference checkout)")
        _L = C.CDLL(str(_SO))
        for name in dir(_L):
            pass
        _L.refcpu_max_threads.restype = C.c_int
        _L.refcpu_sizeof_simparams.restype = C.c_int
    return _L


def _p(a):
    # data_as keeps a reference to the array, so temporaries live through the call
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def set_threads(n: int) -> None:
    lib().refcpu_set_threads(int(n))


def max_threads() -> int:
    return int(lib().refcpu_max_threads())


def morton30(pos4, mn4, mx4):
    pos4 = _f32(pos4)
    n = len(pos4)
    codes = np.zeros(n, np.uint32)
    idx = np.zeros(n, np.int32)
    lib().refcpu_morton30(_p(pos4), n, _p(_f32(mn4)), _p(_f32(mx4)), _p(codes), _p(idx))
    return codes, idx


def aabb(pos4):
    pos4 = _f32(pos4)
    mn, mx = np.zeros(4, np.float32), np.zeros(4, np.float32)
    lib().refcpu_aabb(_p(pos4), len(pos4), _p(mn), _p(mx))
    return mn, mx


def sort_pairs_u32(keys, vals):
    k, v = _u32(keys).copy(), _u32(vals).copy()
    lib().refcpu_sort_pairs_u32(_p(k), _p(v), C.c_long(len(k)))
    return k, v


def radix_tree(sorted_codes):
    codes = _u32(sorted_codes)
    n = len(codes)
    m = max(2 * n - 1, 1)
    t = {"is_leaf": np.zeros(m, np.uint8), "left": np.full(m, -1, np.int32),
         "right": np.full(m, -1, np.int32), "parent": np.full(m, -1, np.int32),
         "min_r": np.full(m, -1, np.int32), "max_r": np.full(m, -1, np.int32)}
    lib().refcpu_radix_tree(_p(codes), n, _p(t["is_leaf"]), _p(t["left"]), _p(t["right"]),
                            _p(t["parent"]), _p(t["min_r"]), _p(t["max_r"]))
    return t


def leaves_and_refit(tree, sorted_idx, pos4, r):
    n = len(sorted_idx)
    cms = np.zeros((n, 4), np.float32)
    bounds = np.zeros((max(2 * n - 1, 1), 8), np.float32)
    radii = np.zeros(n, np.float32)
    L = lib()
    L.refcpu_leaf_nodes(n, _p(tree["is_leaf"]), _p(tree["left"]), _p(tree["right"]),
                        _p(tree["parent"]), _p(tree["min_r"]), _p(tree["max_r"]), _p(cms),
                        _p(bounds), _p(_i32(sorted_idx)), _p(radii), _p(_f32(pos4)),
                        C.c_float(r))
    leaf_bounds = bounds.copy()
    L.refcpu_internal_nodes(n, _p(tree["left"]), _p(tree["right"]), _p(tree["parent"]),
                            _p(bounds))
    return cms, leaf_bounds, bounds, radii


def calc_hash(params, pos4):
    pos4 = _f32(pos4)
    n = len(pos4)
    h = np.zeros(n, np.uint32)
    idx = np.zeros(n, np.uint32)
    lib().refcpu_calc_hash(C.byref(params), _p(pos4), n, _p(h), _p(idx))
    return h, idx


def reorder(shash, sidx, pos4, vel4, num_cells):
    n = len(shash)
    cs = np.zeros(num_cells, np.uint32)
    ce = np.zeros(num_cells, np.uint32)
    sp = np.zeros((n, 4), np.float32)
    sv = np.zeros((n, 4), np.float32)
    lib().refcpu_reorder(_p(cs), _p(ce), _p(sp), _p(sv), _p(_u32(shash)), _p(_u32(sidx)),
                         _p(_f32(pos4)), _p(_f32(vel4)), n, C.c_long(num_cells))
    return cs, ce, sp, sv


def collide_grid_dem(params, rb_idx, spos4, svel4, rel4, gidx, cstart, cend):
    n = len(spos4)
    pf = np.zeros((n, 4), np.float32)
    pt = np.zeros((n, 4), np.float32)
    lib().refcpu_collide_grid_dem(C.byref(params), _p(_i32(rb_idx)), _p(pf), _p(pt),
                                  _p(_f32(spos4)), _p(_f32(svel4)), _p(_f32(rel4)),
                                  _p(_u32(gidx)), _p(_u32(cstart)), _p(_u32(cend)), n)
    return pf, pt


def reduce_impulses(pf4, pt4, vel4, ang4, mass, ib9, counts):
    v, a = _f32(vel4).copy(), _f32(ang4).copy()
    lib().refcpu_reduce_impulses(_p(_f32(pf4)), _p(_f32(pt4)), _p(v), _p(a), _p(_f32(mass)),
                                 _p(_f32(ib9)), _p(_i32(counts)), len(counts), len(pf4))
    return v, a


def gpu_integrator(params, dt, state):
    s = {k: _f32(v).copy() for k, v in state.items()}
    nb = len(s["cms"])
    lib().refcpu_gpu_integrator(_p(s["cms"]), _p(s["vel"]), _p(s["ang"]), _p(s["quat"]),
                                _p(s["ib"]), _p(s["cur"]), _p(s["model"]), _p(s["cum"]),
                                C.c_float(dt), _p(_f32(np.ones(nb))), nb, C.byref(params))
    return s


def global_attributes(cms4, rbvel4, rbang4, quat4, rb_idx, rel4):
    n, nb = len(rel4), len(cms4)
    q, rel = _f32(quat4).copy(), _f32(rel4).copy()
    pos, vel = np.zeros((n, 4), np.float32), np.zeros((n, 4), np.float32)
    lib().refcpu_global_attributes(_p(_f32(cms4)), _p(_f32(rbvel4)), _p(rel), _p(pos), _p(vel),
                                   _p(q), _p(_f32(rbang4)), _p(_i32(rb_idx)), n, nb)
    return rel, pos, vel, q


def collide_static_scene(params, spos4, svel4, rel4, scene_spos4, scene_normals4, gidx,
                         scene_gidx, cstart, cend, lin4, ang4):
    """FindAndHandleAugmentedRealityCollisionsUniformGridKernel; returns updated (linear,
    angular, color)."""
    n = len(spos4)
    lin, ang = _f32(lin4).copy(), _f32(ang4).copy()
    color = np.zeros((len(lin), 4), np.float32)
    lib().refcpu_collide_static_scene(C.byref(params), _p(lin), _p(ang), _p(color),
                                      _p(_f32(spos4)), _p(_f32(svel4)), _p(_f32(rel4)),
                                      _p(_f32(scene_spos4)), _p(_f32(scene_normals4)),
                                      _p(_u32(gidx)), _p(_u32(scene_gidx)), _p(_u32(cstart)),
                                      _p(_u32(cend)), n)
    return lin, ang, color


def collide_bvh_rigid(params, rb_idx, rel4, vel4, tree, cms4, bounds8, sorted_idx, radii):
    n = len(sorted_idx)
    pf = np.zeros((n, 4), np.float32)
    pt = np.zeros((n, 4), np.float32)
    pp = np.zeros((n, 4), np.float32)
    lib().refcpu_collide_bvh_rigid(C.byref(params), _p(pf), _p(_i32(rb_idx)), _p(pp),
                                   _p(_f32(rel4)), _p(pt), _p(_f32(vel4).copy()),
                                   _p(tree["is_leaf"]), _p(tree["left"]), _p(tree["right"]),
                                   _p(tree["min_r"]), _p(tree["max_r"]), _p(_f32(cms4)),
                                   _p(_f32(bounds8)), _p(_i32(sorted_idx)), _p(_f32(radii)), n)
    return pf, pt, pp


def find_rb_collisions_bvh(params, rb_idx, tree, cms4, bounds8, sorted_idx, radii, cd0):
    n = len(sorted_idx)
    cd = _f32(cd0).copy()
    cp = np.zeros(n, np.int32)
    cb = np.zeros(n, np.int32)
    lib().refcpu_find_rb_collisions_bvh(C.byref(params), _p(_i32(rb_idx)), _p(tree["is_leaf"]),
                                        _p(tree["left"]), _p(tree["right"]), _p(tree["min_r"]),
                                        _p(tree["max_r"]), _p(_f32(cms4)), _p(_f32(bounds8)),
                                        _p(_i32(sorted_idx)), _p(_f32(radii)), n, _p(cd), _p(cp),
                                        _p(cb))
    return cd, cp, cb


def find_rb_collisions_grid(params, rb_idx, spos4, gidx, cstart, cend, cd0):
    """FindRigidBodyCollisionsUniformGridKernel -> (distance, body, particle) per original index."""
    n = len(spos4)
    cd = _f32(cd0).copy()
    cb = np.zeros(n, np.int32)
    cp = np.zeros(n, np.int32)
    lib().refcpu_find_rb_collisions_grid(C.byref(params), _p(_i32(rb_idx)), _p(_f32(spos4)),
                                         _p(_u32(gidx)), _p(_u32(cstart)), _p(_u32(cend)), n,
                                         _p(cd), _p(cb), _p(cp))
    return cd, cb, cp


def wall_collisions(ppos4, rbpos4, mn3, mx3, rbvel4, rbang4, ib9, mass, rb_idx, counts, radius):
    v, a = _f32(rbvel4).copy(), _f32(rbang4).copy()
    lib().refcpu_wall_collisions(_p(_f32(ppos4)), _p(_f32(rbpos4)), _p(_f32(mn3)),
                                 _p(_f32(mx3)), _p(v), _p(a), _p(_f32(ib9)), _p(_f32(mass)),
                                 _p(_i32(rb_idx)), _p(_i32(counts)), len(counts), len(ppos4),
                                 C.c_float(radius))
    return v, a


def integrate_momentum(params, state, dt, radii, mass, mn3, mx3):
    s = {k: _f32(v).copy() for k, v in state.items()}
    nb = len(s["cms"])
    lib().refcpu_integrate_momentum(*[_p(s[k]) for k in ("cms", "vel", "force", "ang", "quat",
                                                        "torque", "angmom", "linmom", "ib", "cur",
                                                        "acc")],
                                    C.c_float(dt), _p(_f32(radii)), _p(_f32(mass)),
                                    _p(_f32(mn3)), _p(_f32(mx3)), nb, C.byref(params))
    return s


def integrate_particles(params, pos4, vel4, rb_idx, dt, mn3, mx3):
    p, v = _f32(pos4).copy(), _f32(vel4).copy()
    lib().refcpu_integrate_particles(C.byref(params), _p(p), _p(v), _p(_i32(rb_idx).copy()), len(p),
                                     C.c_float(dt), _p(_f32(mn3)), _p(_f32(mx3)))
    return p, v


def collide_particles(params, rb_idx, rel4, spos4, svel4, gidx, cstart, cend, vel_out=None):
    n = len(spos4)
    pf = np.zeros((n, 4), np.float32)
    pt = np.zeros((n, 4), np.float32)
    nv = np.zeros((n, 4), np.float32) if vel_out is None else _f32(vel_out).copy()
    lib().refcpu_collide_particles(C.byref(params), _p(pf), _p(_i32(rb_idx)), _p(_f32(rel4)),
                                   _p(pt), _p(nv), _p(_f32(spos4)), _p(_f32(svel4)),
                                   _p(_u32(gidx)), _p(_u32(cstart)), _p(_u32(cend)), n)
    return pf, pt, nv


def sis_step(params, rb_idx, offsets, cms4, vel4, ang4, inertia9, mass, rel4, contact_distance,
             contact_body, contact_particle, scene_normals4=None, solve=True):
    """GatherRigidBodyCollisions (or GatherAugmentedRealityCollisions when scene_normals4 is
    given) followed by SequentialImpulseSolver -- the reference's own host loops
    (Particles/updateFunctions.cpp:1431-1874) on a stand-in ParticleSystem.  Returns the
    contact list (normal, point, body1, body2, bias, the accumulated impulse and the two
    accumulated frictions after the solve), the bodies' new velocity and angular velocity,
    and the re-posed particles (rel, pos, particle velocity) of the solver's tail."""
    n, nb = len(rb_idx), len(cms4)
    counts = np.diff(_i32(offsets)).astype(np.int32)
    cms, vel, ang = _f32(cms4).copy(), _f32(vel4).copy(), _f32(ang4).copy()
    ib, m = _f32(inertia9).copy(), _f32(mass).copy()
    rel = _f32(rel4).copy()
    pos, pvel = np.zeros((n, 4), np.float32), np.zeros((n, 4), np.float32)
    quat = np.tile(np.array([0, 0, 0, 1], np.float32), (nb, 1))
    cd = _f32(contact_distance).copy()
    cb = _i32(contact_body if contact_body is not None else np.zeros(n)).copy()
    cp = _i32(contact_particle).copy()
    sn = None if scene_normals4 is None else _f32(scene_normals4)
    cap = n
    out = {"normal": np.zeros((cap, 4), np.float32), "point": np.zeros((cap, 4), np.float32),
           "body1": np.zeros(cap, np.int32), "body2": np.zeros(cap, np.int32),
           "bias": np.zeros(cap, np.float32), "acc": np.zeros((cap, 3), np.float32)}
    L = lib()
    L.refcpu_sis_step.restype = C.c_int
    k = L.refcpu_sis_step(C.byref(params), nb, n, _p(counts), _p(cms), _p(vel), _p(ang), _p(ib),
                          _p(m), _p(rel), _p(pos), _p(pvel), _p(quat), _p(_i32(rb_idx).copy()),
                          _p(cd), _p(cb), _p(cp), _p(sn), 0 if sn is None else len(sn),
                          int(sn is not None), int(solve), cap, _p(out["normal"]),
                          _p(out["point"]), _p(out["body1"]), _p(out["body2"]), _p(out["bias"]),
                          _p(out["acc"]))
    res = {key: v[:k] for key, v in out.items()}
    res.update({"vel": vel, "ang": ang, "rel": rel, "pos": pos, "pvel": pvel, "count": k})
    return res


def init_object(path, model: str, scale: float, radius: float):
    """ParticleSystem::initObject's body set-up (RigidBodies/RigidBodyAddition.cpp:1576-1756) on
    a particle-body file -> (centred offsets [N, 3], inverse inertia [9], glm::mat3 order)."""
    from pathlib import Path as _P
    text = _P(path).read_bytes()
    n = int(text.split(b"\n", 1)[0].split()[0])
    rel = np.zeros((n, 4), np.float32)
    inv = np.zeros(9, np.float32)
    L = lib()
    L.refcpu_init_object.restype = C.c_int
    got = L.refcpu_init_object(C.c_char_p(text), C.c_char_p(model.encode()), C.c_float(scale),
                               C.c_float(radius), _p(rel), _p(inv))
    assert got == n
    return rel[:, :3].copy(), inv


def ar_collide_impulse(params, rb_idx, rel4, inertia9, mass, scene_radii, spos4, svel4,
                       scene_spos4, scene_normals4, gidx, scene_gidx, cstart, cend, new_vel4):
    """ARcollisionsUniformGridKernel (Kernels/RB_UniformGridKernels.cu:590-678) -> per-particle
    force, torque, impulse count, colour, and new_vel4 (free particles)."""
    n = len(spos4)
    count = np.zeros(n, np.int32)
    pf, pt, color = (np.zeros((n, 4), np.float32) for _ in range(3))
    nv = _f32(new_vel4).copy()
    lib().refcpu_ar_collide_impulse(C.byref(params), _p(count), _p(pf), _p(_i32(rb_idx)),
                                    _p(_f32(rel4)), _p(pt), _p(_f32(inertia9)), _p(_f32(mass)),
                                    _p(color), _p(_f32(scene_radii)), _p(nv), _p(_f32(spos4)),
                                    _p(_f32(svel4)), _p(_f32(scene_spos4)),
                                    _p(_f32(scene_normals4)), _p(_u32(gidx)),
                                    _p(_u32(scene_gidx)), _p(_u32(cstart)), _p(_u32(cend)), n)
    return pf, pt, count, color, nv


def ar_find_contacts(params, spos4, scene_spos4, gidx, scene_gidx, cstart, cend,
                     contact_distance, contact_point):
    """FindAugmentedRealityCollisionsUniformGridKernel (:927-1021) -> (distance, point, colour)."""
    n = len(spos4)
    cd = _f32(contact_distance).copy()
    cp = _i32(contact_point).copy()
    color = np.zeros((n, 4), np.float32)
    lib().refcpu_ar_find_contacts(C.byref(params), _p(cp), _p(cd), _p(color), _p(_f32(spos4)),
                                  _p(_f32(scene_spos4)), _p(_u32(gidx)), _p(_u32(scene_gidx)),
                                  _p(_u32(cstart)), _p(_u32(cend)), n)
    return cd, cp, color


def collide_bvh_static(params, rb_idx, rel4, pos4, vel4, tree, cms4, bounds8, sorted_idx, radii,
                       rb_force4, rb_torque4, mass):
    """staticCollideBVHSoARigidBody (Kernels/RB_BVHKernels.cu:293-442), threads run in order
    -> (body force, body torque, velocity, colour)."""
    n, m = len(pos4), len(cms4)
    f, t = _f32(rb_force4).copy(), _f32(rb_torque4).copy()
    vel = _f32(vel4).copy()
    color = np.zeros((n, 4), np.float32)
    lib().refcpu_collide_bvh_static(C.byref(params), _p(color), _p(_f32(pos4)), _p(_f32(rel4)),
                                    _p(t), _p(f), _p(_f32(mass)), _p(_i32(rb_idx)), _p(vel),
                                    _p(tree["is_leaf"]), _p(tree["left"]), _p(tree["right"]),
                                    _p(tree["min_r"]), _p(tree["max_r"]), _p(_f32(cms4)),
                                    _p(_f32(bounds8)), _p(_i32(sorted_idx)), _p(_f32(radii)), n, m)
    return f, t, vel, color


def find_contacts_bvh_static(params, pos4, tree, cms4, bounds8, sorted_idx, radii,
                             contact_distance, contact_point):
    """FindAugmentedRealityCollisionsBVHKernel (Kernels/RB_BVHKernels.cu:920-1023) ->
    (distance, point, colour)."""
    n, m = len(pos4), len(cms4)
    cd, cp = _f32(contact_distance).copy(), _i32(contact_point).copy()
    color = np.zeros((n, 4), np.float32)
    lib().refcpu_find_contacts_bvh_static(C.byref(params), _p(color), _p(_f32(pos4)),
                                          _p(tree["is_leaf"]), _p(tree["left"]),
                                          _p(tree["right"]), _p(tree["min_r"]),
                                          _p(tree["max_r"]), _p(_f32(cms4)), _p(_f32(bounds8)),
                                          _p(_i32(sorted_idx)), _p(_f32(radii)), n, m, _p(cd),
                                          _p(cp))
    return cd, cp, color


def range_image(depth, camera16, radius):
    """RGBDloader and computeNormals (Kernels/customRangeImageLoader.cu:14-177) over the grid
    loadRangeImage launches (whole 16 x 32 blocks) -> pos4, radii, vao5, norm4; pixels the
    reference does not write stay NaN."""
    d = np.ascontiguousarray(depth, dtype=np.uint16)
    h, w = d.shape
    pos4 = np.full((h * w, 4), np.nan, np.float32)
    radii = np.full(h * w, np.nan, np.float32)
    vao5 = np.full((h * w, 5), np.nan, np.float32)
    norm4 = np.full((h * w, 4), np.nan, np.float32)
    cam = _f32(np.asarray(camera16, np.float32).reshape(16))
    lib().refcpu_range_cloud(_p(d), C.c_int(w), C.c_int(h), _p(cam), C.c_float(radius),
                             _p(pos4), _p(radii), _p(vao5))
    lib().refcpu_range_normals(_p(pos4), C.c_int(w), C.c_int(h), _p(norm4))
    return {"pos4": pos4, "radii": radii, "vao5": vao5, "norm4": norm4}
