"""numpy wrappers over oracle/liboracle.so -- the CPU restatement used as the checker.

TEST INFRASTRUCTURE ONLY: imported by tests/, bench.py (cpu_baseline and reference arm) and
__graft_entry__.smoke(); never by the product package.
"""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

import numpy as np

from . import build as _build

_SO = Path(__file__).resolve().parent / "liboracle.so"
if not _SO.exists():
    _build.build()
_L = C.CDLL(str(_SO))


def _p(a: np.ndarray | None):
    # data_as keeps a reference to the array, so temporaries live through the call
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


for _name in ["or_aabb", "or_morton30", "or_morton63", "or_sort_pairs_u32", "or_sort_pairs_u64",
              "or_radix_tree_u32", "or_radix_tree_u64", "or_leaves", "or_refit",
              "or_collide_bvh_dem", "or_find_contacts_bvh", "or_calc_hash", "or_reorder",
              "or_collide_grid_dem", "or_reduce_bodies", "or_reduce_impulses",
              "or_integrate_reference", "or_global_attributes", "or_walls_reference"]:
    getattr(_L, _name).restype = None
_L.or_pairs_brute.restype = C.c_long
_L.or_step.restype = C.c_int
_L.or_step_ex.restype = C.c_int
_L.or_step_f64.restype = C.c_int
for _name in ["or_aabb", "or_morton30", "or_morton63", "or_sort_pairs_u32", "or_sort_pairs_u64",
              "or_calc_hash", "or_reorder", "or_collide_grid_dem", "or_pairs_brute"]:
    pass  # argument conversion is explicit at each call (longs passed via C.c_long)


# ---- stages -------------------------------------------------------------------------------------
def aabb(pos4):
    pos4 = _f32(pos4)
    mn, mx = np.zeros(4, np.float32), np.zeros(4, np.float32)
    _L.or_aabb(_p(pos4), C.c_long(len(pos4)), _p(mn), _p(mx))
    return mn, mx


def morton30(pos4, mn4, mx4) -> np.ndarray:
    pos4, mn4, mx4 = _f32(pos4), _f32(mn4), _f32(mx4)
    out = np.zeros(len(pos4), np.uint32)
    _L.or_morton30(_p(pos4), C.c_long(len(pos4)), _p(mn4), _p(mx4), _p(out))
    return out


def morton63(pos4, mn4, mx4) -> np.ndarray:
    pos4, mn4, mx4 = _f32(pos4), _f32(mn4), _f32(mx4)
    out = np.zeros(len(pos4), np.uint64)
    _L.or_morton63(_p(pos4), C.c_long(len(pos4)), _p(mn4), _p(mx4), _p(out))
    return out


def sort_pairs(keys, vals=None, begin_bit=0, end_bit=None):
    """Stable sort by key bits [begin, end) -- cub::DeviceRadixSort::SortPairs order."""
    keys = np.ascontiguousarray(keys)
    n = len(keys)
    vin = None if vals is None else _u32(vals)
    vout = np.zeros(n, np.uint32)
    if keys.dtype == np.uint64:
        kout = np.zeros(n, np.uint64)
        _L.or_sort_pairs_u64(_p(keys), _p(vin), _p(kout), _p(vout), C.c_long(n), begin_bit,
                             64 if end_bit is None else end_bit)
    else:
        keys = _u32(keys)
        kout = np.zeros(n, np.uint32)
        _L.or_sort_pairs_u32(_p(keys), _p(vin), _p(kout), _p(vout), C.c_long(n), begin_bit,
                             32 if end_bit is None else end_bit)
    return kout, vout


def radix_tree(sorted_codes) -> dict[str, np.ndarray]:
    codes = np.ascontiguousarray(sorted_codes)
    n = len(codes)
    m = max(2 * n - 1, 1)
    t = {"is_leaf": np.zeros(m, np.uint8), "left": np.full(m, -1, np.int32),
         "right": np.full(m, -1, np.int32), "parent": np.full(m, -1, np.int32),
         "min_r": np.full(m, -1, np.int32), "max_r": np.full(m, -1, np.int32)}
    fn = _L.or_radix_tree_u64 if codes.dtype == np.uint64 else _L.or_radix_tree_u32
    if codes.dtype != np.uint64:
        codes = _u32(codes)
    fn(_p(codes), n, _p(t["is_leaf"]), _p(t["left"]), _p(t["right"]), _p(t["parent"]),
       _p(t["min_r"]), _p(t["max_r"]))
    return t


def leaves(tree: dict, sorted_idx, pos4, r: float):
    n = len(sorted_idx)
    sorted_idx, pos4 = _i32(sorted_idx), _f32(pos4)
    cms = np.zeros((n, 4), np.float32)
    bounds = np.zeros((max(2 * n - 1, 1), 8), np.float32)
    _L.or_leaves(n, _p(sorted_idx), _p(pos4), C.c_float(r), _p(tree["is_leaf"]),
                 _p(tree["min_r"]), _p(tree["max_r"]), _p(cms), _p(bounds))
    return cms, bounds


def refit(tree: dict, bounds: np.ndarray) -> np.ndarray:
    n = (len(tree["left"]) + 1) // 2
    b = _f32(bounds).copy()
    _L.or_refit(n, _p(tree["left"]), _p(tree["right"]), _p(b))
    return b


def collide_bvh_dem(prm4, rb_idx, rel4, vel4, tree, cms4, bounds8, sorted_idx, radii):
    n = len(sorted_idx)
    pf = np.zeros((n, 4), np.float32)
    pt = np.zeros((n, 4), np.float32)
    pp = np.zeros((n, 4), np.float32)
    args = [_f32(prm4), _i32(rb_idx), _f32(rel4), _f32(vel4), tree["is_leaf"], tree["left"],
            tree["right"], _f32(cms4), _f32(bounds8), _i32(sorted_idx), _f32(radii)]
    _L.or_collide_bvh_dem(*[_p(a) for a in args], n, _p(pf), _p(pt), _p(pp))
    return pf, pt, pp


def find_contacts_bvh(rb_idx, tree, cms4, bounds8, sorted_idx, radii, contact_distance):
    n = len(sorted_idx)
    cd = _f32(contact_distance).copy()
    cp = np.zeros(n, np.int32)
    cb = np.zeros(n, np.int32)
    args = [_i32(rb_idx), tree["is_leaf"], tree["left"], tree["right"], tree["max_r"],
            _f32(cms4), _f32(bounds8), _i32(sorted_idx), _f32(radii)]
    _L.or_find_contacts_bvh(*[_p(a) for a in args], n, _p(cd), _p(cp), _p(cb))
    return cd, cp, cb


def pairs_brute(pos4, rb_idx, two_r: float) -> np.ndarray:
    pos4, rb_idx = _f32(pos4), _i32(rb_idx)
    n = len(pos4)
    cnt = _L.or_pairs_brute(_p(pos4), _p(rb_idx), n, C.c_float(two_r), None, C.c_long(0))
    out = np.zeros((max(cnt, 1), 2), np.int32)
    _L.or_pairs_brute(_p(pos4), _p(rb_idx), n, C.c_float(two_r), _p(out), C.c_long(cnt))
    return out[:cnt]


def calc_hash(origin, cell, dims, pos4) -> np.ndarray:
    g6 = _f32(list(origin) + list(np.broadcast_to(cell, 3)))
    d3 = _u32(dims)
    pos4 = _f32(pos4)
    out = np.zeros(len(pos4), np.uint32)
    _L.or_calc_hash(_p(g6), _p(d3), _p(pos4), C.c_long(len(pos4)), _p(out))
    return out


def reorder(shash, sidx, pos4, vel4, num_cells: int):
    n = len(shash)
    cs = np.zeros(num_cells, np.uint32)
    ce = np.zeros(num_cells, np.uint32)
    sp = np.zeros((n, 4), np.float32)
    sv = np.zeros((n, 4), np.float32)
    _L.or_reorder(_p(_u32(shash)), _p(_u32(sidx)), _p(_f32(pos4)), _p(_f32(vel4)), C.c_long(n),
                  C.c_long(num_cells), _p(cs), _p(ce), _p(sp), _p(sv))
    return cs, ce, sp, sv


def collide_grid_dem(origin, cell, dims, prm5, rb_idx, spos4, svel4, rel4, gidx, cstart, cend,
                     pf0=None, pt0=None):
    n = len(spos4)
    g6 = _f32(list(origin) + list(np.broadcast_to(cell, 3)))
    pf = np.zeros((n, 4), np.float32) if pf0 is None else _f32(pf0).copy()
    pt = np.zeros((n, 4), np.float32) if pt0 is None else _f32(pt0).copy()
    args = [g6, _u32(dims), _f32(prm5), _i32(rb_idx), _f32(spos4), _f32(svel4), _f32(rel4),
            _u32(gidx), _u32(cstart), _u32(cend)]
    _L.or_collide_grid_dem(*[_p(a) for a in args], C.c_long(n), _p(pf), _p(pt))
    return pf, pt


def reduce_bodies(pf4, pt4, offsets):
    nb = len(offsets) - 1
    bf = np.zeros((nb, 4), np.float32)
    bt = np.zeros((nb, 4), np.float32)
    _L.or_reduce_bodies(_p(_f32(pf4)), _p(_f32(pt4)), _p(_i32(offsets)), nb, _p(bf), _p(bt))
    return bf, bt


def reduce_impulses(pf4, pt4, offsets, vel4, ang4, mass, ib9):
    nb = len(offsets) - 1
    v, a = _f32(vel4).copy(), _f32(ang4).copy()
    _L.or_reduce_impulses(_p(_f32(pf4)), _p(_f32(pt4)), _p(_i32(offsets)), nb, _p(v), _p(a),
                          _p(_f32(mass)), _p(_f32(ib9)))
    return v, a


def integrate_reference(gravity, w_damping, dt, state: dict) -> dict:
    s = {k: _f32(v).copy() for k, v in state.items()}
    nb = len(s["cms"])
    _L.or_integrate_reference(_p(_f32(gravity)), C.c_float(w_damping), C.c_float(dt), nb,
                              _p(s["cms"]), _p(s["vel"]), _p(s["ang"]), _p(s["quat"]),
                              _p(s["ib"]), _p(s["cur"]), _p(s.get("model")), _p(s.get("cum")))
    return s


def global_attributes(cms4, rbvel4, rbang4, quat4, rb_idx, rel4):
    n, nb = len(rel4), len(cms4)
    q, rel = _f32(quat4).copy(), _f32(rel4).copy()
    pos, vel = np.zeros((n, 4), np.float32), np.zeros((n, 4), np.float32)
    _L.or_global_attributes(n, nb, _p(_f32(cms4)), _p(_f32(rbvel4)), _p(_f32(rbang4)), _p(q),
                            _p(_i32(rb_idx)), _p(rel), _p(pos), _p(vel))
    return rel, pos, vel, q


def walls_reference(radius, ppos4, rbpos4, mn3, mx3, rbvel4, rbang4, ib9, mass, rb_idx, offsets):
    v, a = _f32(rbvel4).copy(), _f32(rbang4).copy()
    nb = len(offsets) - 1
    _L.or_walls_reference(C.c_float(radius), _p(_f32(ppos4)), _p(_f32(rbpos4)), _p(_f32(mn3)),
                          _p(_f32(mx3)), _p(v), _p(a), _p(_f32(ib9)), _p(_f32(mass)),
                          _p(_i32(rb_idx)), _p(_i32(offsets)), nb)
    return v, a


# ---- the fused PHYSICAL step ---------------------------------------------------------------------
def _next_pow2(v: int) -> int:
    p = 1
    while p < v and p < (1 << 31):
        p <<= 1
    return p


def scene_grid(scene, cell_size: float | None = None, grid_log2=None):
    """The grid the library gives a scene (same rule as the C++ scene set-up)."""
    c = np.float32(cell_size if cell_size else (scene.cell_size or 2 * np.float32(scene.radius)))
    g = list(scene.grid_log2 if grid_log2 is None else grid_log2)
    origin = [float(x) for x in scene.box_min]
    dims = []
    for a in range(3):
        if g[a] > 0:
            dims.append(1 << int(g[a]))
        else:
            ext = float(scene.box_max[a]) - float(scene.box_min[a])
            cells = int(math.ceil(ext / float(c)))
            dims.append(max(4, _next_pow2(max(cells, 1))))
    if not any(x > 0 for x in g):
        cap = max(1 << 12, _next_pow2(8 * max(scene.num_particles, 1)))
        while dims[0] * dims[1] * dims[2] > cap:
            a = int(np.argmax(dims))
            if dims[a] <= 4:
                break
            dims[a] >>= 1
    return origin, [float(c)] * 3, dims


def _scene_arrays(scene):
    rel = _f32(scene.particle_rel).copy()
    rel[:, 3] = scene.body_index().view(np.float32)
    s15 = _f32(list(scene.box_min) + list(scene.box_max) + list(scene.gravity) +
               [scene.radius, scene.dt, scene.spring, scene.damping, scene.shear,
                scene.attraction])
    return rel, s15


def step(scene, steps: int = 1, grid=None, state: dict | None = None,
         broadphase: str = "grid", cloud=None) -> dict:
    """Float32 restatement of ar_step (operation for operation).  Returns the new body state
    and, for the last step, the sorted keys / indices, per-particle forces and body sums.
    broadphase 'bvh' restates the BVH step (sorted keys are then the 30-bit Morton codes).
    cloud = (positions [M, 4], normals [M, 4]): a static point cloud attached to the scene
    (ar_scene_set_static_cloud; grid broad phase)."""
    if broadphase == "bvh":
        assert cloud is None, "a static cloud needs the grid broad phase"
        return _step_bvh(scene, steps, state)
    origin, cell, dims = grid if grid is not None else scene_grid(scene)
    rel, s15 = _scene_arrays(scene)
    st = state or {"pos": scene.body_pos, "quat": scene.body_quat, "vel": scene.body_vel,
                   "angvel": scene.body_angvel}
    st = {k: _f32(v).copy() for k, v in st.items()}
    n, nb = scene.num_particles, scene.num_bodies
    out = {"skeys": np.zeros(n, np.uint32), "sidx": np.zeros(n, np.uint32),
           "pforce": np.zeros((n, 4), np.float32), "bforce": np.zeros((nb, 4), np.float32),
           "btorque": np.zeros((nb, 4), np.float32)}
    g6 = _f32(list(origin) + list(cell))
    cp = cn = None
    cm = 0
    if cloud is not None:
        cp, cn = _f32(cloud[0]).reshape(-1, 4), _f32(cloud[1]).reshape(-1, 4)
        assert cp.shape == cn.shape
        cm = cp.shape[0]
    ok = _L.or_step_ex(_p(s15), _p(g6), _p(_u32(dims)), nb, n, _p(st["pos"]), _p(st["quat"]),
                       _p(st["vel"]), _p(st["angvel"]), _p(_f32(scene.body_mass)),
                       _p(_f32(scene.body_inv_inertia)), _p(_i32(scene.body_offsets)), _p(rel),
                       steps, _p(out["skeys"]), _p(out["sidx"]), _p(out["pforce"]),
                       _p(out["bforce"]), _p(out["btorque"]), _p(cp), _p(cn), cm)
    st.update(out)
    st["finite"] = bool(ok)
    return st


_L.or_step_bvh.restype = C.c_int


def _step_bvh(scene, steps: int, state: dict | None) -> dict:
    rel, s15 = _scene_arrays(scene)
    st = state or {"pos": scene.body_pos, "quat": scene.body_quat, "vel": scene.body_vel,
                   "angvel": scene.body_angvel}
    st = {k: _f32(v).copy() for k, v in st.items()}
    n, nb = scene.num_particles, scene.num_bodies
    out = {"skeys": np.zeros(n, np.uint64), "sidx": np.zeros(n, np.uint32),
           "pforce": np.zeros((n, 4), np.float32), "bforce": np.zeros((nb, 4), np.float32),
           "btorque": np.zeros((nb, 4), np.float32)}
    ok = _L.or_step_bvh(_p(s15), nb, n, _p(st["pos"]), _p(st["quat"]), _p(st["vel"]),
                        _p(st["angvel"]), _p(_f32(scene.body_mass)),
                        _p(_f32(scene.body_inv_inertia)), _p(_i32(scene.body_offsets)), _p(rel),
                        steps, _p(out["skeys"]), _p(out["sidx"]), _p(out["pforce"]),
                        _p(out["bforce"]), _p(out["btorque"]))
    st.update(out)
    st["finite"] = bool(ok)
    return st


def step_f64(scene, steps: int = 1, state: dict | None = None, cell: float | None = None) -> dict:
    """FP64 restatement of the same physics (contacts decided in double)."""
    rel = np.ascontiguousarray(scene.particle_rel, np.float64).copy()
    rel[:, 3] = scene.body_index()
    s15 = np.ascontiguousarray(list(scene.box_min) + list(scene.box_max) + list(scene.gravity) +
                               [scene.radius, scene.dt, scene.spring, scene.damping,
                                scene.shear, scene.attraction], np.float64)
    c = float(cell or scene_grid(scene)[1][0])
    cell3 = np.array([c, c, c], np.float64)
    st = state or {"pos": scene.body_pos, "quat": scene.body_quat, "vel": scene.body_vel,
                   "angvel": scene.body_angvel}
    st = {k: np.ascontiguousarray(v, np.float64).copy() for k, v in st.items()}
    n, nb = scene.num_particles, scene.num_bodies
    pf = np.zeros((n, 4), np.float64)
    bf = np.zeros((nb, 4), np.float64)
    bt = np.zeros((nb, 4), np.float64)
    ok = _L.or_step_f64(_p(s15), _p(cell3), nb, n, _p(st["pos"]), _p(st["quat"]), _p(st["vel"]),
                        _p(st["angvel"]), _p(np.ascontiguousarray(scene.body_mass, np.float64)),
                        _p(np.ascontiguousarray(scene.body_inv_inertia, np.float64)),
                        _p(_i32(scene.body_offsets)), _p(rel), steps, _p(pf), _p(bf), _p(bt))
    st.update({"pforce": pf, "bforce": bf, "btorque": bt, "finite": bool(ok)})
    return st


# ---- remaining reference stages ------------------------------------------------------------------
_L.or_integrate_momentum.restype = None
_L.or_integrate_particles.restype = None
_L.or_collide_grid_particles.restype = None
_L.or_reduce_rbvars.restype = C.c_int


def integrate_momentum(state: dict, dt, radii, mass, mn3, mx3, gravity, bdamp, gdamp) -> dict:
    """integrateRigidBody.  state keys: cms vel force ang quat torque angmom linmom ib cur acc."""
    s = {k: _f32(v).copy() for k, v in state.items()}
    nb = len(s["cms"])
    _L.or_integrate_momentum(*[_p(s[k]) for k in ("cms", "vel", "force", "ang", "quat", "torque",
                                                 "angmom", "linmom", "ib", "cur", "acc")],
                             C.c_float(dt), _p(_f32(radii)), _p(_f32(mass)), _p(_f32(mn3)),
                             _p(_f32(mx3)), _p(_f32(gravity)), C.c_float(bdamp), C.c_float(gdamp), nb)
    return s


def integrate_particles(pos4, vel4, rb_idx, dt, mn3, mx3, gravity, gdamp, bdamp, r):
    p, v = _f32(pos4).copy(), _f32(vel4).copy()
    _L.or_integrate_particles(_p(p), _p(v), _p(_i32(rb_idx)), len(p), C.c_float(dt), _p(_f32(mn3)),
                              _p(_f32(mx3)), _p(_f32(gravity)), C.c_float(gdamp), C.c_float(bdamp),
                              C.c_float(r))
    return p, v


def collide_grid_particles(origin, cell, dims, prm5, rb_idx, spos4, svel4, rel4, gidx, cstart,
                           cend, vel_out=None):
    n = len(spos4)
    g6 = _f32(list(origin) + list(np.broadcast_to(cell, 3)))
    pf = np.zeros((n, 4), np.float32)
    pt = np.zeros((n, 4), np.float32)
    nv = np.zeros((n, 4), np.float32) if vel_out is None else _f32(vel_out).copy()
    args = [g6, _u32(dims), _f32(prm5), _i32(rb_idx), _f32(spos4), _f32(svel4), _f32(rel4),
            _u32(gidx), _u32(cstart), _u32(cend)]
    _L.or_collide_grid_particles(*[_p(a) for a in args], C.c_long(n), _p(pf), _p(pt), _p(nv))
    return pf, pt, nv


def reduce_rigid_body_variables(pf4, pt4, starts, counts, bf4, bt4):
    bf, bt = _f32(bf4).copy(), _f32(bt4).copy()
    ok = _L.or_reduce_rbvars(_p(_f32(pf4)), _p(_f32(pt4)), _p(_i32(starts)), _p(_i32(counts)),
                             len(starts), _p(bf), _p(bt))
    return bf, bt, bool(ok)


_L.or_collide_static_scene.restype = None


def collide_static_scene(origin, cell, dims, radius, prm4, spos4, svel4, rel4, scene_spos4,
                         scene_normals4, gidx, scene_gidx, cstart, cend, lin4, ang4):
    """FindAndHandleAugmentedRealityCollisionsUniformGridKernel; returns updated (linear,
    angular, color)."""
    n = len(spos4)
    lin, ang = _f32(lin4).copy(), _f32(ang4).copy()
    color = np.zeros((len(lin), 4), np.float32)
    g6 = _f32(list(origin) + list(cell))
    _L.or_collide_static_scene(_p(g6), _p(_u32(dims)), C.c_float(radius), _p(_f32(prm4)),
                               _p(_f32(spos4)), _p(_f32(svel4)), _p(_f32(rel4)),
                               _p(_f32(scene_spos4)), _p(_f32(scene_normals4)), _p(_u32(gidx)),
                               _p(_u32(scene_gidx)), _p(_u32(cstart)), _p(_u32(cend)), n,
                               _p(lin), _p(ang), _p(color))
    return lin, ang, color



# ---- sequential-impulse path ---------------------------------------------------------------------
_L.or_find_contacts_grid.restype = None
_L.or_gather_contacts.restype = C.c_long
_L.or_sequential_impulse.restype = None


def find_contacts_grid(origin, cell, dims, radius, rb_idx, spos4, gidx, cstart, cend,
                       contact_distance=None):
    """FindRigidBodyCollisionsUniformGridKernel on sorted arrays -> (distance, body, particle)
    per original particle index (distance starts at contact_distance, default 0)."""
    n = len(spos4)
    g6 = _f32(list(origin) + list(np.broadcast_to(cell, 3)))
    cd = np.zeros(n, np.float32) if contact_distance is None else _f32(contact_distance).copy()
    cb = np.zeros(n, np.int32)
    cp = np.zeros(n, np.int32)
    _L.or_find_contacts_grid(_p(g6), _p(_u32(dims)), C.c_float(radius), _p(_i32(rb_idx)),
                             _p(_f32(spos4)), _p(_u32(gidx)), _p(_u32(cstart)), _p(_u32(cend)),
                             C.c_long(n), _p(cd), _p(cb), _p(cp))
    return cd, cb, cp


def gather_contacts(radius, restitution, rb_idx, cms4, vel4, ang4, rel4, contact_distance,
                    colliding_body, colliding_particle) -> dict:
    """GatherRigidBodyCollisions: the contact list in particle order."""
    n = len(rb_idx)
    out = {"normal": np.zeros((n, 4), np.float32), "point": np.zeros((n, 4), np.float32),
           "body1": np.zeros(n, np.int32), "body2": np.zeros(n, np.int32),
           "bias": np.zeros(n, np.float32)}
    c = _L.or_gather_contacts(C.c_float(radius), C.c_float(restitution), C.c_long(n),
                              _p(_i32(rb_idx)), _p(_f32(cms4)), _p(_f32(vel4)), _p(_f32(ang4)),
                              _p(_f32(rel4)), _p(_f32(contact_distance)),
                              _p(_i32(colliding_body)), _p(_i32(colliding_particle)),
                              _p(out["normal"]), _p(out["point"]), _p(out["body1"]),
                              _p(out["body2"]), _p(out["bias"]))
    return {k: v[:c] for k, v in out.items()}


def sequential_impulse(contacts: dict, cms4, vel4, ang4, inertia9, mass, iterations=18,
                       ar_friction=0.3, rb_friction=0.1, gravity_y=-9.81, acc=None):
    """SequentialImpulseSolver as the reference's host loop -> (vel4, ang4, accumulated
    impulse, friction, friction 2)."""
    k = len(contacts["body1"])
    vel, ang = _f32(vel4).copy(), _f32(ang4).copy()
    if acc is None:
        acc = tuple(np.zeros(k, np.float32) for _ in range(3))
    a0, a1, a2 = (_f32(a).copy() for a in acc)
    _L.or_sequential_impulse(C.c_long(k), _p(_f32(contacts["normal"])), _p(_f32(contacts["point"])),
                             _p(_i32(contacts["body1"])), _p(_i32(contacts["body2"])),
                             _p(_f32(contacts["bias"])), _p(a0), _p(a1), _p(a2), _p(_f32(cms4)),
                             _p(vel), _p(ang), _p(_f32(inertia9)), _p(_f32(mass)),
                             C.c_int(iterations), C.c_float(ar_friction), C.c_float(rb_friction),
                             C.c_float(gravity_y))
    return vel, ang, a0, a1, a2


def sis_solve(state: dict, rb_idx, origin, cell, dims, radius, restitution=1.0,
              ar_friction=0.3, rb_friction=0.1, gravity_y=-9.81e-3, iterations=18) -> dict:
    """The second half of an updateUniformGridSIS step on a snapshot taken after the
    integration: hash, sort, reorder, contact search, gather, SequentialImpulseSolver, and
    computeGlobalAttributes with the (identity) step rotation."""
    pos, pvel = _f32(state["pos"]), _f32(state["pvel"])
    n = len(pos)
    h = calc_hash(origin, cell, dims, pos)
    sh, si = sort_pairs(h, np.arange(n, dtype=np.uint32))
    cs, ce, sp, sv = reorder(sh, si, pos, pvel, int(np.prod(dims)))
    cd, cb, cp = find_contacts_grid(origin, cell, dims, radius, rb_idx, sp, si, cs, ce)
    contacts = gather_contacts(radius, restitution, rb_idx, state["cms"], state["vel"],
                               state["ang"], state["rel"], cd, cb, cp)
    vel, ang, a0, a1, a2 = sequential_impulse(contacts, state["cms"], state["vel"], state["ang"],
                                              state["cur"], state["mass"], iterations,
                                              ar_friction, rb_friction, gravity_y)
    rel, ppos, ppvel, _ = global_attributes(state["cms"], vel, ang, state["quat"], rb_idx,
                                            state["rel"])
    return {"vel": vel, "ang": ang, "rel": rel, "pos": ppos, "pvel": ppvel,
            "contacts": len(contacts["body1"]), "acc": a0}


# ---- static scene: impulse variant, deepest contacts, contact gather -------------------------
_L.or_ar_collide_impulse.restype = None
_L.or_ar_find_contacts.restype = None
_L.or_gather_static_contacts.restype = C.c_long


def ar_collide_impulse(origin, cell, dims, radius, restitution, rb_idx, rel4, inertia9, mass,
                       scene_radii, spos4, svel4, scene_spos4, gidx, scene_gidx, cstart, cend,
                       new_vel4=None):
    """ARcollisionsUniformGridKernel -> (force, torque, count, colour, new_vel4)."""
    n = len(spos4)
    g6 = _f32(list(origin) + [cell] * 3)
    pf, pt, color = (np.zeros((n, 4), np.float32) for _ in range(3))
    count = np.zeros(n, np.int32)
    nv = np.zeros((n, 4), np.float32) if new_vel4 is None else _f32(new_vel4).copy()
    _L.or_ar_collide_impulse(_p(g6), _p(_u32(dims)), C.c_float(radius), C.c_float(restitution),
                             _p(_i32(rb_idx)), _p(_f32(rel4)), _p(_f32(inertia9)),
                             _p(_f32(mass)), _p(_f32(scene_radii)), _p(_f32(spos4)),
                             _p(_f32(svel4)), _p(_f32(scene_spos4)), _p(_u32(gidx)),
                             _p(_u32(scene_gidx)), _p(_u32(cstart)), _p(_u32(cend)), n, _p(pf),
                             _p(pt), _p(count), _p(nv), _p(color))
    return pf, pt, count, color, nv


def ar_find_contacts(origin, cell, dims, radius, spos4, scene_spos4, gidx, scene_gidx, cstart,
                     cend, contact_distance, contact_point):
    """FindAugmentedRealityCollisionsUniformGridKernel -> (distance, point, colour)."""
    n = len(spos4)
    g6 = _f32(list(origin) + [cell] * 3)
    cd, cp = _f32(contact_distance).copy(), _i32(contact_point).copy()
    color = np.zeros((n, 4), np.float32)
    _L.or_ar_find_contacts(_p(g6), _p(_u32(dims)), C.c_float(radius), _p(_f32(spos4)),
                           _p(_f32(scene_spos4)), _p(_u32(gidx)), _p(_u32(scene_gidx)),
                           _p(_u32(cstart)), _p(_u32(cend)), n, _p(cd), _p(cp), _p(color))
    return cd, cp, color


def gather_static_contacts(restitution, rb_idx, cms4, vel4, ang4, rel4, scene_normals4,
                           contact_distance, contact_point) -> dict:
    """GatherAugmentedRealityCollisions: the contact list in particle order."""
    n = len(rb_idx)
    out = {"normal": np.zeros((n, 4), np.float32), "point": np.zeros((n, 4), np.float32),
           "body1": np.zeros(n, np.int32), "body2": np.zeros(n, np.int32),
           "bias": np.zeros(n, np.float32)}
    c = _L.or_gather_static_contacts(C.c_float(restitution), C.c_long(n), _p(_i32(rb_idx)),
                                     _p(_f32(cms4)), _p(_f32(vel4)), _p(_f32(ang4)),
                                     _p(_f32(rel4)), _p(_f32(scene_normals4)),
                                     _p(_f32(contact_distance)), _p(_i32(contact_point)),
                                     _p(out["normal"]), _p(out["point"]), _p(out["body1"]),
                                     _p(out["body2"]), _p(out["bias"]))
    return {k: v[:c] for k, v in out.items()}


_L.or_collide_bvh_static.restype = None
_L.or_find_contacts_bvh_static.restype = None


def collide_bvh_static(prm4, radius, rb_idx, rel4, pos4, vel4, tree, cms4, bounds8, radii):
    """staticCollideBVHSoARigidBody -> (force, torque, velocity, colour), per particle."""
    n, m = len(pos4), len(cms4)
    pf, pt, color = (np.zeros((n, 4), np.float32) for _ in range(3))
    vel = _f32(vel4).copy()
    _L.or_collide_bvh_static(_p(_f32(prm4)), C.c_float(radius), _p(_i32(rb_idx)), _p(_f32(rel4)),
                             _p(_f32(pos4)), _p(vel), _p(tree["is_leaf"]), _p(_i32(tree["left"])),
                             _p(_i32(tree["right"])), _p(_f32(cms4)), _p(_f32(bounds8)),
                             _p(_f32(radii)), m, n, _p(pf), _p(pt), _p(color))
    return pf, pt, vel, color


def find_contacts_bvh_static(radius, pos4, tree, cms4, bounds8, sorted_idx, radii,
                             contact_distance, contact_point):
    """FindAugmentedRealityCollisionsBVHKernel -> (distance, point, colour)."""
    n, m = len(pos4), len(cms4)
    cd, cp = _f32(contact_distance).copy(), _i32(contact_point).copy()
    color = np.zeros((n, 4), np.float32)
    _L.or_find_contacts_bvh_static(C.c_float(radius), _p(_f32(pos4)), _p(tree["is_leaf"]),
                                   _p(_i32(tree["left"])), _p(_i32(tree["right"])),
                                   _p(_f32(cms4)), _p(_f32(bounds8)), _p(_i32(sorted_idx)),
                                   _p(_f32(radii)), m, n, _p(cd), _p(cp), _p(color))
    return cd, cp, color


def range_image_cloud(depth: np.ndarray, camera16, radius: float, with_vao: bool = True):
    """RGBDloader (Kernels/customRangeImageLoader.cu:14-113): depth [h, w] uint16 -> pos4 [h*w, 4],
    radii [h*w], vao5 [h*w, 5]; pixels past the reference's bound stay NaN."""
    d = np.ascontiguousarray(depth, dtype=np.uint16)
    h, w = d.shape
    pos4 = np.full((h * w, 4), np.nan, np.float32)
    radii = np.full(h * w, np.nan, np.float32)
    vao5 = np.full((h * w, 5), np.nan, np.float32) if with_vao else None
    cam = _f32(np.asarray(camera16, np.float32).reshape(16))
    _L.or_range_cloud(_p(d), C.c_int(w), C.c_int(h), _p(cam), C.c_float(radius), _p(pos4),
                      _p(radii), _p(vao5) if with_vao else None)
    return {"pos4": pos4, "radii": radii, "vao5": vao5}


def range_image_normals(pos4: np.ndarray, w: int, h: int, init: float = np.nan):
    """computeNormals (Kernels/customRangeImageLoader.cu:122-177); border pixels keep `init`."""
    norm4 = np.full((h * w, 4), init, np.float32)
    _L.or_range_normals(_p(_f32(pos4)), C.c_int(w), C.c_int(h), _p(norm4))
    return norm4
