"""ctypes binding of libarsim.so (the C ABI declared in include/arsim.h).

The shared library is built in-tree by ``diploma_thesis_b200.build``; importing this module
without it raises immediately -- there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libarsim.so"

AR_OK = 0
STATUS_NAMES = {0: "AR_OK", 1: "AR_ERR_INVALID_ARG", 2: "AR_ERR_OOM", 3: "AR_ERR_TIMEOUT",
                4: "AR_ERR_NAN", 5: "AR_ERR_CUDA", 6: "AR_ERR_UNSUPPORTED",
                7: "AR_ERR_OVERFLOW"}
AR_BROADPHASE_GRID = 0
AR_BROADPHASE_BVH = 1


class ArError(RuntimeError):
    def __init__(self, status: int, where: str, message: str):
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class SimParams(C.Structure):
    """Byte-compatible with the reference's SimParams (Kernels/particleSystem.cuh:27-55)."""
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


class SceneDesc(C.Structure):
    _fields_ = [("num_bodies", C.c_int), ("num_particles", C.c_int), ("radius", C.c_float),
                ("box_min", C.c_float * 3), ("box_max", C.c_float * 3),
                ("gravity", C.c_float * 3), ("dt", C.c_float), ("spring", C.c_float),
                ("damping", C.c_float), ("shear", C.c_float), ("attraction", C.c_float),
                ("broadphase", C.c_int), ("cell_size", C.c_float), ("grid_log2", C.c_int * 3),
                ("block_size", C.c_int)]


class SceneInit(C.Structure):
    _fields_ = [("body_pos4", C.c_void_p), ("body_quat4", C.c_void_p),
                ("body_vel4", C.c_void_p), ("body_angvel4", C.c_void_p),
                ("body_mass", C.c_void_p), ("body_inv_inertia9", C.c_void_p),
                ("body_offsets", C.c_void_p), ("particle_rel4", C.c_void_p)]


class ServerStatsC(C.Structure):
    """ar_server_stats (include/arsim.h)."""
    _fields_ = [("completed", C.c_int), ("offered", C.c_int), ("peak_resident", C.c_int),
                ("ticks", C.c_int), ("wall_s", C.c_double), ("scene_steps", C.c_longlong),
                ("particle_steps", C.c_longlong), ("peak_bytes", C.c_size_t),
                ("host_admit_s", C.c_double), ("host_set_s", C.c_double),
                ("host_step_s", C.c_double), ("host_retire_s", C.c_double),
                ("host_wait_s", C.c_double)]


class SceneView(C.Structure):
    _fields_ = [("num_bodies", C.c_int), ("num_particles", C.c_int),
                ("body_pos4", C.c_void_p), ("body_quat4", C.c_void_p),
                ("body_vel4", C.c_void_p), ("body_angvel4", C.c_void_p),
                ("body_mass", C.c_void_p), ("body_inv_inertia9", C.c_void_p),
                ("body_offsets", C.c_void_p), ("particle_rel4", C.c_void_p),
                ("body_force4", C.c_void_p), ("body_torque4", C.c_void_p)]


AR_MAX_BATCH_CELLS = (1 << 32) - 1
AR_MAX_BATCH_PARTICLES = (1 << 30) - 1


class StepView(C.Structure):
    _fields_ = [("num_particles", C.c_int), ("num_cells", C.c_uint64), ("key_bits", C.c_int),
                ("sorted_keys", C.c_void_p), ("sorted_idx", C.c_void_p),
                ("sorted_pos4", C.c_void_p), ("sorted_vel4", C.c_void_p),
                ("particle_force4", C.c_void_p), ("cells2", C.c_void_p),
                ("key_bytes", C.c_int), ("broadphase", C.c_int), ("tree_left", C.c_void_p),
                ("tree_right", C.c_void_p), ("tree_parent", C.c_void_p),
                ("tree_nodes16", C.c_void_p)]


P = C.c_void_p
I = C.c_int
F = C.c_float
S = C.c_void_p  # stream

# name -> argtypes (restype is always ar_status / int unless listed in _RESTYPE)
SIGNATURES = {
    "ar_ctx_create": [I, C.POINTER(P)],
    "ar_ctx_destroy": [P],
    "ar_ctx_status": [P, S],
    "ar_ctx_reserve": [P, C.c_size_t],
    "ar_last_error": [],
    "ar_version": [],
    "ar_test_fail_allocations": [C.c_long],
    "ar_scene_aabb": [P, P, I, P, P, S],
    "ar_morton30": [P, P, I, P, P, P, P, S],
    "ar_morton30_box": [P, P, I, C.POINTER(F), C.POINTER(F), P, P, S],
    "ar_morton63": [P, P, I, P, P, P, P, S],
    "ar_radix_sort_pairs_u32": [P, P, P, P, P, I, I, I, S],
    "ar_radix_sort_pairs_u64": [P, P, P, P, P, I, I, I, S],
    "ar_radix_sort_pairs_u32_noalloc": [P, P, P, P, I, I, I, P, S],
    "ar_radix_sort_pairs_u32_ex": [P, P, P, P, P, I, I, I, C.c_uint32, S],
    "ar_lbvh_build": [P, P, I, P, P, P, P, P, P, S],
    "ar_lbvh_build64": [P, P, I, P, P, P, P, P, P, S],
    "ar_lbvh_leaves": [P, I, P, P, F, P, P, P, P, P, P, S],
    "ar_lbvh_refit": [P, I, P, P, P, P, S],
    "ar_collide_bvh_dem": [P, C.POINTER(SimParams), P, P, P, P, P, P, P, P, P, P, P, I, P, P, P, S],
    "ar_find_contacts_bvh": [P, P, P, P, P, P, P, P, P, P, P, I, P, P, P, S],
    "ar_pairs_bvh": [P, F, P, P, P, P, P, P, P, P, I, P, I, P, S],
    "ar_pairs_grid": [P, C.POINTER(SimParams), P, P, P, P, P, I, P, I, P, S],
    "ar_calc_hash": [P, C.POINTER(SimParams), P, I, P, P, S],
    "ar_reorder_cells": [P, P, P, P, P, I, C.c_uint32, P, P, P, P, S],
    "ar_collide_grid_dem": [P, C.POINTER(SimParams), P, P, P, P, P, P, P, I, P, P, S],
    "ar_range_image_cloud": [P, P, I, I, P, F, P, P, P, S],
    "ar_range_image_normals": [P, P, I, I, P, S],
    "ar_collide_static_scene_dem": [P, C.POINTER(SimParams), P, P, P, P, P, P, P, P, P, I, P, P, P, S],
    "ar_collide_static_scene_impulse": [P, C.POINTER(SimParams), P, P, P, P, P, P, P, P, P, P, P,
                                        P, I, P, P, P, P, P, S],
    "ar_find_contacts_static_scene": [P, C.POINTER(SimParams), P, P, P, P, P, P, I, P, P, P, S],
    "ar_collide_bvh_static": [P, C.POINTER(SimParams), P, P, P, P, P, P, P, P, P, P, P, I, I, P,
                              P, P, S],
    "ar_find_contacts_bvh_static": [P, C.POINTER(SimParams), P, P, P, P, P, P, P, P, P, I, I, P,
                                    P, P, S],
    "ar_gather_static_contacts": [P, C.POINTER(SimParams), I, P, P, P, P, P, P, P, P, I, P, P, P,
                                  P, P, P, P, P, P, S],
    "ar_reduce_bodies": [P, P, P, P, I, P, P, S],
    "ar_reduce_impulses": [P, P, P, P, I, P, P, P, P, S],
    "ar_integrate_reference": [P, C.POINTER(SimParams), F, I, P, P, P, P, P, P, P, P, P, S],
    "ar_global_attributes": [P, I, I, P, P, P, P, P, P, P, P, S],
    "ar_reset_quaternions": [P, P, I, S],
    "ar_integrate_momentum": [P, C.POINTER(SimParams), F, I, P, P, P, P, P, P, P, P, P, P, P, P,
                              P, C.POINTER(F), C.POINTER(F), S],
    "ar_integrate_particles": [P, C.POINTER(SimParams), F, P, P, P, I, C.POINTER(F),
                               C.POINTER(F), S],
    "ar_fill_f32": [P, P, C.c_long, F, S],
    "ar_collide_grid_particles": [P, C.POINTER(SimParams), P, P, P, P, P, P, P, I, P, P, P, S],
    "ar_reduce_rigid_body_variables": [P, P, P, P, P, I, P, P, S],
    "ar_walls_reference": [P, F, P, P, C.POINTER(F), C.POINTER(F), P, P, P, P, P, P, I, I, S],
    "ar_scene_create": [P, C.POINTER(SceneDesc), C.POINTER(SceneInit), S, C.POINTER(P)],
    "ar_scene_destroy": [P],
    "ar_scene_footprint": [C.POINTER(SceneDesc)],
    "ar_scene_cells": [C.POINTER(SceneDesc)],
    "ar_scene_destroy_async": [P, S],
    "ar_scene_set_static_cloud": [P, P, P, P, I, S],
    "ar_batch_set_scenes_limited": [P, C.POINTER(P), I, P],
    "ar_batch_model_matrices": [P, P, S],
    "ar_scene_model_matrices": [P, P, S],
    "ar_scene_download": [P, P, P, P, P, S],
    "ar_scene_download_async": [P, P, P, P, P, S],
    "ar_scene_upload": [P, P, P, P, P, S],
    "ar_find_contacts_grid": [P, P, P, P, P, P, P, I, P, P, P, S],
    "ar_gather_contacts": [P, P, I, P, P, P, P, P, P, P, P, I, P, P, P, P, P, P, P, P, P, S],
    "ar_sequential_impulse": [P, P, P, I, P, P, P, P, P, P, P, P, I, P, P, P, P, P, I, S],
    "ar_scene_upload_state": [P, P, S],
    "ar_scene_download_state": [P, P, S],
    "ar_scene_download_state_async": [P, P, S],
    "ar_step_profile": [P, P, I, C.POINTER(F), S],
    "ar_batch_profile": [P, P, I, C.POINTER(F), S],
    "ar_scene_get_view": [P, C.POINTER(SceneView)],
    "ar_scene_grid_info": [P, C.POINTER(F), C.POINTER(F), C.POINTER(C.c_uint32)],
    "ar_scene_step_view": [P, C.POINTER(StepView)],
    "ar_step": [P, P, I, I, S],
    "ar_scene_particle_forces": [P, P, P, S],
    "ar_batch_create": [P, C.POINTER(P)],
    "ar_batch_destroy": [P],
    "ar_batch_set_scenes": [P, C.POINTER(P), I],
    "ar_batch_step": [P, P, I, I, S],
    "ar_batch_launches_per_step": [P],
    "ar_scene_launches_per_step": [P],
}
_RESTYPE = {"ar_last_error": C.c_char_p, "ar_version": C.c_char_p,
            "ar_scene_footprint": C.c_size_t, "ar_scene_cells": C.c_uint64,
            "ar_batch_launches_per_step": C.c_int,
            "ar_scene_launches_per_step": C.c_int}


def load(path: Path = LIB_PATH) -> C.CDLL:
    if not path.exists():
        raise ImportError(
            f"{path} is missing: build it with `python -m diploma_thesis_b200.build` "
            "(there is no CPU fallback)")
    lib = C.CDLL(str(path))
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPE.get(name, C.c_int)
    return lib


lib = load()


def check(status: int, where: str) -> None:
    if status != AR_OK:
        msg = lib.ar_last_error()
        raise ArError(status, where, msg.decode() if msg else "")


def call(name: str, *args) -> None:
    check(getattr(lib, name)(*args), name)
