// Host driver for the reference's own kernel bodies ("ref_cpu").
//
// TEST INFRASTRUCTURE ONLY (oracle).  Built by oracle/ref_build.py into
// oracle/_ref/libref_cpu.so; loaded only by tests/, bench.py's reference arm and
// __graft_entry__.smoke() as a checker or as the timed CPU baseline.
//
// The kernel bodies come verbatim from the reference checkout (oracle/_ref/extracted.inc,
// generated at build time, never committed) plus the reference's BVHSoAKernels.cu and
// BVHAuxiliary.cuh included from their place in the checkout.  This file only supplies:
//   * an emulated launch: every kernel runs once per (blockIdx, threadIdx) of the grid the
//     reference wrapper would launch, in an OpenMP loop;
//   * host restatements of the three pieces of the reference path that are not kernel
//     bodies: the CUB radix sorts (stable LSD order, restated as a stable LSD sort with the
//     same key-bit treatment), the CUB float4 inclusive scans (restated as the sequential
//     float scan the reference's own DEBUG_SCAN check uses, UniformGridDEM.cu:559-588), and
//     reorderDataAndFindCellStartD (shared memory + __syncthreads, particleKernels.cu:193-258,
//     restated as its sequential neighbour compare);
//   * extern "C" entry points with plain pointers for ctypes.
#include "ref_prelude.h"

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;

#include "BVHAuxiliary.cuh"

#ifndef GLM_FORCE_CUDA
#define GLM_FORCE_CUDA
#endif
#include <glm/glm.hpp>
#include <glm/gtc/quaternion.hpp>

#include <thrust/tuple.h>

// Kernels/particleKernels.cu:42 keeps the parameters in __constant__ memory.
SimParams params;

#include "BVHSoAKernels.cu"
#include "extracted.inc"

#include <omp.h>
#include <algorithm>
#include <cstring>
#include <vector>

namespace {

int g_threads = 0;  // 0 = OpenMP default

template <class F>
void launch(long n_threads, int block, bool parallel, F&& body) {
  long nb = (n_threads + block - 1) / block;
  if (nb < 1) nb = 1;
  const long total = nb * (long)block;
  const int nt = g_threads > 0 ? g_threads : omp_get_max_threads();
#pragma omp parallel for schedule(static) if (parallel) num_threads(nt)
  for (long t = 0; t < total; ++t) {
    blockIdx = make_uint3((unsigned)(t / block), 0, 0);
    threadIdx = make_uint3((unsigned)(t % block), 0, 0);
    blockDim = dim3(block);
    gridDim = dim3((unsigned)nb);
    body();
  }
}

// Stable LSD radix sort of (key, value) pairs over all key bits: the order
// cub::DeviceRadixSort::SortPairs produces (keys ascending, equal keys in input order).
template <class K, class V>
void stable_lsd(K* keys, V* vals, long n) {
  std::vector<K> k2(n);
  std::vector<V> v2(n);
  K* ka = keys; V* va = vals; K* kb = k2.data(); V* vb = v2.data();
  const int passes = (int)sizeof(K);
  for (int p = 0; p < passes; ++p) {
    const int shift = 8 * p;
    long cnt[257] = {0};
    for (long i = 0; i < n; ++i) cnt[((ka[i] >> shift) & 0xFF) + 1]++;
    if (cnt[1 + ((ka[0] >> shift) & 0xFF)] == n && n > 0) continue;  // digit constant
    for (int d = 0; d < 256; ++d) cnt[d + 1] += cnt[d];
    for (long i = 0; i < n; ++i) {
      long dst = cnt[(ka[i] >> shift) & 0xFF]++;
      kb[dst] = ka[i];
      vb[dst] = va[i];
    }
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  if (ka != keys) {
    std::memcpy(keys, ka, n * sizeof(K));
    std::memcpy(vals, va, n * sizeof(V));
  }
}

// CUB's unsigned image of a float key (sign-magnitude flipped to two's-complement order).
inline uint32_t float_key_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

}  // namespace

extern "C" {

void refcpu_set_threads(int n) { g_threads = n; }
int refcpu_max_threads(void) { return g_threads > 0 ? g_threads : omp_get_max_threads(); }
int refcpu_sizeof_simparams(void) { return (int)sizeof(SimParams); }
int refcpu_sizeof_aabb(void) { return (int)sizeof(AABB); }

// ---- Morton codes: generateMortonCodes (BVHSource/BVHkernels.cu:694-716) ----------------
void refcpu_morton30(const float* pos4, int n, const float* min4, const float* max4,
                     uint32_t* codes, int32_t* idx) {
  float4 mn = make_float4(min4[0], min4[1], min4[2], min4[3]);
  float4 mx = make_float4(max4[0], max4[1], max4[2], max4[3]);
  launch(n, 128, true, [&] {
    generateMortonCodes((float4*)pos4, codes, idx, n, mn, mx);
  });
}

// ---- scene AABB: findAABBCub (BVHSource/createMortonCodes.cu:65-107) ---------------------
// Restated: CUB reduces with CustomMin4/CustomMax4 over all four lanes starting from
// (float)0x7f800000 / -(float)0x7f800000 (the `inf` macro is an int, :10).
void refcpu_aabb(const float* pos4, int n, float* min4, float* max4) {
  float lo[4], hi[4];
  for (int c = 0; c < 4; ++c) { lo[c] = (float)0x7f800000; hi[c] = -(float)0x7f800000; }
  for (long i = 0; i < n; ++i)
    for (int c = 0; c < 4; ++c) {
      float v = pos4[4 * i + c];
      lo[c] = (v < lo[c]) ? v : lo[c];
      hi[c] = (v > hi[c]) ? v : hi[c];
    }
  for (int c = 0; c < 4; ++c) { min4[c] = lo[c]; max4[c] = hi[c]; }
}

// ---- CUB DeviceRadixSort::SortPairs (all key bits, stable) -----------------------------
void refcpu_sort_pairs_u32(uint32_t* keys, uint32_t* vals, long n) { stable_lsd(keys, vals, n); }
void refcpu_sort_pairs_u64(uint64_t* keys, uint32_t* vals, long n) { stable_lsd(keys, vals, n); }

// ---- Karras radix tree: kernelConstructRadixTreeSoA (BVHSource/BVHSoAKernels.cu:7-99) --
void refcpu_radix_tree(const uint32_t* sorted_codes, int n, uint8_t* is_leaf, int* left,
                       int* right, int* parent, int* min_r, int* max_r) {
  if (n < 2) return;
  launch(n - 1, 128, true, [&] {
    kernelConstructRadixTreeSoA(n - 1, (bool*)is_leaf, left, right, parent, min_r, max_r,
                                (unsigned int*)sorted_codes);
  });
}

// ---- leaves: initializeRadii + kernelConstructLeafNodesSoA (BVHSoAKernels.cu:108-138) --
void refcpu_leaf_nodes(int n, uint8_t* is_leaf, int* left, int* right, int* parent,
                       int* min_r, int* max_r, float* cms4, void* bounds,
                       const int* sorted_idx, float* radii, const float* pos4, float r) {
  for (int i = 0; i < n; ++i) radii[i] = r;  // initializeRadii (particleKernels.cu:694-701)
  launch(n, 128, true, [&] {
    kernelConstructLeafNodesSoA(n, (bool*)is_leaf, left, right, parent, min_r, max_r,
                                (float4*)cms4, (AABB*)bounds, (int*)sorted_idx, radii,
                                (float4*)pos4, r);
  });
}

// ---- refit: kernelConstructInternalNodesSoA (BVHSoAKernels.cu:148-176) -------------------
// Run on one thread: the reference has no fence between the counter and the child reads,
// so only a serial run gives its intended result deterministically.
void refcpu_internal_nodes(int n, int* left, int* right, int* parent, void* bounds) {
  if (n < 2) return;
  std::vector<int> counters(n - 1, 0);
  launch(n, 128, false, [&] {
    kernelConstructInternalNodesSoA(n, left, right, parent, (AABB*)bounds, counters.data());
  });
}

// ---- grid hash: calcHashD (Kernels/particleKernels.cu:170-189) ---------------------------
void refcpu_calc_hash(const void* sim_params, const float* pos4, int n, uint32_t* hash,
                      uint32_t* idx) {
  std::memcpy(&params, sim_params, sizeof(SimParams));
  launch(n, 512, true, [&] { calcHashD(hash, idx, (float4*)pos4, (uint)n); });
}

// ---- reorderDataAndFindCellStart (particleKernelWrappers.cu:213-254 + kernel :193-258) --
// Restated: cellStart memset to 0xffffffff over all cells, then the neighbour compare.
void refcpu_reorder(uint32_t* cell_start, uint32_t* cell_end, float* sorted_pos4,
                    float* sorted_vel4, const uint32_t* hash, const uint32_t* idx,
                    const float* pos4, const float* vel4, int n, long num_cells) {
  std::memset(cell_start, 0xff, num_cells * sizeof(uint32_t));
  for (int i = 0; i < n; ++i) {
    uint32_t h = hash[i];
    if (i == 0 || h != hash[i - 1]) {
      cell_start[h] = i;
      if (i > 0) cell_end[hash[i - 1]] = i;
    }
    if (i == n - 1) cell_end[h] = i + 1;
    std::memcpy(sorted_pos4 + 4l * i, pos4 + 4l * idx[i], 16);
    std::memcpy(sorted_vel4 + 4l * i, vel4 + 4l * idx[i], 16);
  }
}

// ---- DEM grid collide: FindAndHandleRigidBodyCollisionsUniformGridKernel
//      (RigidBodies/UniformGridDEM.cu:133-204).  pForce/pTorque are accumulated (+=).
void refcpu_collide_grid_dem(const void* sim_params, const int* rb_idx, float* p_force4,
                             float* p_torque4, const float* sorted_pos4,
                             const float* sorted_vel4, const float* rel4,
                             const uint32_t* grid_idx, const uint32_t* cell_start,
                             const uint32_t* cell_end, int n) {
  SimParams p;
  std::memcpy(&p, sim_params, sizeof(SimParams));
  std::vector<float4> color(n);
  float3 zero = make_float3(0, 0, 0);
  launch(n, 128, true, [&] {
    FindAndHandleRigidBodyCollisionsUniformGridKernel(
        (int*)rb_idx, (float4*)p_force4, (float4*)p_torque4, color.data(),
        (float4*)sorted_pos4, (float4*)sorted_vel4, (float4*)rel4, zero, zero,
        (uint*)grid_idx, (uint*)cell_start, (uint*)cell_end, (uint)n, p);
  });
}

// ---- FindAndHandleAugmentedRealityCollisionsUniformGridKernel (UniformGridDEM.cu:243-377) --
// The static scene's particles are sorted into their own grid (cell_start/cell_end over the
// scene's sorted order); impulses are added to p_linear4 / p_angular4 in place.
void refcpu_collide_static_scene(const void* sim_params, float* p_linear4, float* p_angular4,
                                 float* color4, const float* sorted_pos4,
                                 const float* sorted_vel4, const float* rel4,
                                 const float* scene_sorted_pos4, const float* scene_normals4,
                                 const uint32_t* grid_idx, const uint32_t* scene_grid_idx,
                                 const uint32_t* cell_start, const uint32_t* cell_end, int n) {
  SimParams p;
  std::memcpy(&p, sim_params, sizeof(SimParams));
  launch(n, 128, true, [&] {
    FindAndHandleAugmentedRealityCollisionsUniformGridKernel(
        (float4*)p_linear4, (float4*)p_angular4, (float4*)color4, (float4*)sorted_pos4,
        (float4*)sorted_vel4, (float4*)rel4, (float4*)scene_sorted_pos4, (float4*)scene_normals4,
        (uint*)grid_idx, (uint*)scene_grid_idx, (uint*)cell_start, (uint*)cell_end, (uint)n, p);
  });
}

// ---- static scene, impulse variant: ARcollisionsUniformGridKernel (RB_UniformGridKernels.cu:
// 590-678) and the deepest-contact search FindAugmentedRealityCollisionsUniformGridKernel
// (:927-1021), over the grid their wrappers launch.
void refcpu_ar_collide_impulse(const void* sim_params, int* count, float* p_force4,
                               const int* rb_idx, const float* rel4, float* p_torque4,
                               const float* inertia9, const float* mass, float* color4,
                               const float* scene_radii, float* new_vel4,
                               const float* sorted_pos4, const float* sorted_vel4,
                               const float* scene_sorted_pos4, const float* scene_normals4,
                               const uint32_t* grid_idx, const uint32_t* scene_grid_idx,
                               const uint32_t* cell_start, const uint32_t* cell_end, int n) {
  SimParams p;
  std::memcpy(&p, sim_params, sizeof(SimParams));
  launch(n, 128, true, [&] {
    ARcollisionsUniformGridKernel(count, (float4*)p_force4, (int*)rb_idx, (float4*)rel4,
                                  (float4*)p_torque4, (glm::mat3*)inertia9, (float*)mass,
                                  (float4*)color4, (float*)scene_radii, (float4*)new_vel4,
                                  (float4*)sorted_pos4, (float4*)sorted_vel4,
                                  (float4*)scene_sorted_pos4, (float4*)scene_normals4,
                                  (uint*)grid_idx, (uint*)scene_grid_idx, (uint*)cell_start,
                                  (uint*)cell_end, (uint)n, p);
  });
}

void refcpu_ar_find_contacts(const void* sim_params, int* contact_point, float* contact_distance,
                             float* color4, const float* sorted_pos4,
                             const float* scene_sorted_pos4, const uint32_t* grid_idx,
                             const uint32_t* scene_grid_idx, const uint32_t* cell_start,
                             const uint32_t* cell_end, int n) {
  SimParams p;
  std::memcpy(&p, sim_params, sizeof(SimParams));
  launch(n, 128, true, [&] {
    FindAugmentedRealityCollisionsUniformGridKernel(
        contact_point, contact_distance, nullptr, (float4*)color4, (float4*)sorted_pos4,
        (float4*)scene_sorted_pos4, (uint*)grid_idx, (uint*)scene_grid_idx, (uint*)cell_start,
        (uint*)cell_end, (uint)n, p);
  });
}

// ---- static scene through the scene's BVH: staticCollideBVHSoARigidBody
// (RB_BVHKernels.cu:293-442) and FindAugmentedRealityCollisionsBVHKernel (:920-1023) ---------
void refcpu_collide_bvh_static(const void* sim_params, float* color4, const float* pos4,
                               const float* rel4, float* rb_torque4, float* rb_force4,
                               const float* rb_mass, const int* rb_idx, float* vel4,
                               const uint8_t* is_leaf, const int* left, const int* right,
                               const int* min_r, const int* max_r, const float* cms4,
                               const void* bounds, const int* sorted_idx, const float* radii,
                               int n, int num_scene) {
  SimParams p;
  std::memcpy(&p, sim_params, sizeof(SimParams));
  launch(n, 128, false, [&] {  // the kernel adds to per-body totals: run the threads in order
    staticCollideBVHSoARigidBody((float4*)color4, (float4*)pos4, (float4*)rel4,
                                 (float4*)rb_torque4, (float4*)rb_force4, (float*)rb_mass,
                                 (int*)rb_idx, nullptr, (float4*)vel4, nullptr, (bool*)is_leaf,
                                 (int*)left, (int*)right, (int*)min_r, (int*)max_r,
                                 (float4*)cms4, (AABB*)bounds, (int*)sorted_idx, (float*)radii,
                                 n, num_scene, p);
  });
}

void refcpu_find_contacts_bvh_static(const void* sim_params, float* color4, const float* pos4,
                                     const uint8_t* is_leaf, const int* left, const int* right,
                                     const int* min_r, const int* max_r, const float* cms4,
                                     const void* bounds, const int* sorted_idx,
                                     const float* radii, int n, int num_scene,
                                     float* contact_distance, int* contact_point) {
  SimParams p;
  std::memcpy(&p, sim_params, sizeof(SimParams));
  launch(n, 128, true, [&] {
    FindAugmentedRealityCollisionsBVHKernel(
        (float4*)color4, (float4*)pos4, (bool*)is_leaf, (int*)left, (int*)right, (int*)min_r,
        (int*)max_r, (float4*)cms4, (AABB*)bounds, (int*)sorted_idx, (float*)radii, n,
        num_scene, p, contact_distance, contact_point);
  });
}

// ---- ReducePerParticleImpulses (UniformGridDEM.cu:462-666) with CombineReducedImpulses ---
// The two CUB float4 inclusive scans are restated as sequential float scans.
void refcpu_reduce_impulses(const float* p_force4, const float* p_torque4, float* rb_vel4,
                            float* rb_ang4, const float* rb_mass, const float* rb_inv_inertia9,
                            const int* particles_per_object, int num_bodies, int n) {
  std::vector<float4> lin(n), ang(n);
  float4 a = make_float4(0, 0, 0, 0), b = make_float4(0, 0, 0, 0);
  for (int i = 0; i < n; ++i) {
    a += ((const float4*)p_force4)[i];
    b += ((const float4*)p_torque4)[i];
    lin[i] = a;
    ang[i] = b;
  }
  std::vector<int> cum(num_bodies);
  int run = 0;
  for (int i = 0; i < num_bodies; ++i) { run += particles_per_object[i]; cum[i] = run; }
  launch(num_bodies, 128, true, [&] {
    CombineReducedImpulses(lin.data(), ang.data(), (float4*)rb_vel4, (float4*)rb_ang4,
                           (float*)rb_mass, (glm::mat3*)rb_inv_inertia9, cum.data(), num_bodies);
  });
}

// ---- GPUintegratorKernel (Kernels/rigidBodyKernels.cu:262-348) --------------------------
void refcpu_gpu_integrator(float* cms4, float* vel4, float* ang4, float* quat4,
                           const float* inv_inertia9, float* cur_inertia9, float* model16,
                           float* cum_quat4, float dt, const float* mass, int num_bodies,
                           const void* sim_params) {
  SimParams p;
  std::memcpy(&p, sim_params, sizeof(SimParams));
  launch(num_bodies, 128, true, [&] {
    GPUintegratorKernel((float4*)cms4, (float4*)vel4, (float4*)ang4, (glm::quat*)quat4,
                        (glm::mat3*)inv_inertia9, (glm::mat3*)cur_inertia9,
                        (glm::mat4*)model16, (glm::quat*)cum_quat4, dt, (float*)mass,
                        num_bodies, p);
  });
}

// ---- computeGlobalAttributes + resetQuaternionKernel (rigidBodyKernels.cu:386-456) ------
void refcpu_global_attributes(const float* cms4, const float* rb_vel4, float* rel4,
                              float* pos4, float* vel4, float* quat4, const float* ang4,
                              const int* rb_idx, int n, int num_bodies) {
  launch(n, 128, true, [&] {
    computeGlobalAttributes((float4*)cms4, (float4*)rb_vel4, (float4*)rel4, (float4*)pos4,
                            (float4*)vel4, (glm::quat*)quat4, (float4*)ang4, (int*)rb_idx, n);
  });
  launch(num_bodies, 128, true, [&] { resetQuaternionKernel((glm::quat*)quat4, num_bodies); });
}

// ---- BVH DEM traversal: collideBVHSoARigidBody (Kernels/RB_BVHKernels.cu:100-244) -------
void refcpu_collide_bvh_rigid(const void* sim_params, float* p_force4, const int* rb_idx,
                              float* p_positions4, const float* rel4, float* p_torque4,
                              float* vel4, const uint8_t* is_leaf, const int* left,
                              const int* right, const int* min_r, const int* max_r,
                              const float* cms4, const void* bounds, const int* sorted_idx,
                              const float* radii, int n) {
  SimParams p;
  std::memcpy(&p, sim_params, sizeof(SimParams));
  std::vector<float4> color(n);
  launch(n, 128, true, [&] {
    collideBVHSoARigidBody(color.data(), (float4*)p_force4, (int*)rb_idx,
                           (float4*)p_positions4, nullptr, (float4*)rel4, (float4*)p_torque4,
                           (float4*)vel4, (bool*)is_leaf, (int*)left, (int*)right,
                           (int*)min_r, (int*)max_r, (float4*)cms4, (AABB*)bounds,
                           (int*)sorted_idx, (float*)radii, n, p);
  });
}

// ---- deepest contact per particle: FindRigidBodyCollisionsBVHKernel (:760-876) ----------
void refcpu_find_rb_collisions_bvh(const void* sim_params, const int* rb_idx,
                                   const uint8_t* is_leaf, const int* left, const int* right,
                                   const int* min_r, const int* max_r, const float* cms4,
                                   const void* bounds, const int* sorted_idx,
                                   const float* radii, int n, float* contact_distance,
                                   int* colliding_particle, int* colliding_body) {
  SimParams p;
  std::memcpy(&p, sim_params, sizeof(SimParams));
  std::vector<float4> color(n);
  launch(n, 128, true, [&] {
    FindRigidBodyCollisionsBVHKernel(color.data(), (int*)rb_idx, (bool*)is_leaf, (int*)left,
                                     (int*)right, (int*)min_r, (int*)max_r, (float4*)cms4,
                                     (AABB*)bounds, (int*)sorted_idx, (float*)radii, n, p,
                                     contact_distance, colliding_particle, colliding_body);
  });
}

// ---- deepest contact per particle on the grid: FindRigidBodyCollisionsUniformGridKernel
// (Kernels/RB_UniformGridKernels.cu:731-842) ---------------------------------------------------
void refcpu_find_rb_collisions_grid(const void* sim_params, const int* rb_idx,
                                    const float* sorted_pos4, const uint32_t* grid_idx,
                                    const uint32_t* cell_start, const uint32_t* cell_end, int n,
                                    float* contact_distance, int* colliding_body,
                                    int* colliding_particle) {
  SimParams p;
  std::memcpy(&p, sim_params, sizeof(SimParams));
  std::vector<float4> color(n);
  launch(n, 128, true, [&] {
    FindRigidBodyCollisionsUniformGridKernel((int*)rb_idx, colliding_body, colliding_particle,
                                             contact_distance, color.data(), (float4*)sorted_pos4,
                                             (uint*)grid_idx, (uint*)cell_start, (uint*)cell_end,
                                             (uint)n, p);
  });
}

// ---- integrateRigidBody (Kernels/rigidBodyKernels.cu:40-166) ------------------------------
void refcpu_integrate_momentum(float* cms4, float* vel4, float* force4, float* ang4,
                               float* quat4, float* torque4, float* ang_mom4, float* lin_mom4,
                               const float* inv_inertia9, float* cur9, float* acc3, float dt,
                               const float* radii, const float* mass, const float* mn3,
                               const float* mx3, int nb, const void* sim_params) {
  SimParams p;
  std::memcpy(&p, sim_params, sizeof(SimParams));
  float3 mn = make_float3(mn3[0], mn3[1], mn3[2]), mx = make_float3(mx3[0], mx3[1], mx3[2]);
  launch(nb, 128, true, [&] {
    integrateRigidBody((float4*)cms4, (float4*)vel4, (float4*)force4, (float4*)ang4,
                       (glm::quat*)quat4, (float4*)torque4, (float4*)ang_mom4,
                       (float4*)lin_mom4, (glm::mat3*)inv_inertia9, (glm::mat3*)cur9,
                       (glm::vec3*)acc3, dt, (float*)radii, (float*)mass, mn, mx, nb, p);
  });
}

// ---- integrate_functor through integrateSystem (Kernels/particleKernels.cu:50-148) -------
void refcpu_integrate_particles(const void* sim_params, float* pos4, float* vel4,
                                int* rb_idx, int n, float dt, const float* mn3,
                                const float* mx3) {
  std::memcpy(&params, sim_params, sizeof(SimParams));
  const integrate_functor f(dt, make_float3(mn3[0], mn3[1], mn3[2]),
                            make_float3(mx3[0], mx3[1], mx3[2]));
  for (int i = 0; i < n; ++i) {
    // operator() widens the functor's own box members (particleKernels.cu:78-84); each device
    // thread applies it to its own copy, so each particle gets a fresh copy here too
    integrate_functor g = f;
    thrust::tuple<float4&, float4&, int&> t(((float4*)pos4)[i], ((float4*)vel4)[i], rb_idx[i]);
    g(t);
  }
}

// ---- collideD (Kernels/particleKernels.cu:344-406) ------------------------------------------
void refcpu_collide_particles(const void* sim_params, float* p_force4, const int* rb_idx,
                              const float* rel4, float* p_torque4, float* new_vel4,
                              const float* sorted_pos4, const float* sorted_vel4,
                              const uint32_t* grid_idx, const uint32_t* cell_start,
                              const uint32_t* cell_end, int n) {
  std::memcpy(&params, sim_params, sizeof(SimParams));
  std::vector<float4> color(n);
  launch(n, 128, true, [&] {
    collideD((float4*)p_force4, (int*)rb_idx, (float4*)rel4, (float4*)p_torque4, color.data(),
             (float4*)new_vel4, (float4*)sorted_pos4, (float4*)sorted_vel4, (uint*)grid_idx,
             (uint*)cell_start, (uint*)cell_end, (uint)n);
  });
}

// ---- WallCollisionWrapper (WallCollisions.cu:338-597) ------------------------------------
// The six DetectWallCollisionKernel launches and HandleWallCollisionKernelUnmapped are the
// reference bodies; the host glue (wall planes, the three stable CUB sorts, the prefix of
// particle counts) is restated from the wrapper.
void refcpu_wall_collisions(const float* particle_pos4, const float* rb_pos4,
                            const float* min_pos3, const float* max_pos3, float* rb_vel4,
                            float* rb_ang4, const float* inv_inertia9, const float* rb_mass,
                            const int* rb_idx, const int* particles_per_rb, int num_bodies,
                            int n, float radius) {
  std::vector<float4> cn(n, make_float4(0, 0, 0, 0)), cp(n, make_float4(0, 0, 0, 0)),
      cw(n, make_float4(0, 0, 0, 0));
  std::vector<float> cd(n, 0.0f);
  float3 mn = make_float3(min_pos3[0], min_pos3[1], min_pos3[2]);
  float3 mx = make_float3(max_pos3[0], max_pos3[1], max_pos3[2]);
  float4 unit = make_float4(1, 1, 1, 1);
  const float4 normals[6] = {make_float4(1, 0, 0, 0),  make_float4(0, 1, 0, 0),
                             make_float4(0, 0, 1, 0),  make_float4(-1, 0, 0, 0),
                             make_float4(0, -1, 0, 0), make_float4(0, 0, -1, 0)};
  for (int w = 0; w < 6; ++w) {
    float4 nrm = normals[w];
    float wall_pos;
    if (w < 3) {
      wall_pos = dot(make_float3(nrm), mx);
    } else {
      float sign = dot(nrm, unit);
      wall_pos = dot(make_float3(nrm) * sign, mn);
    }
    launch(n, 128, true, [&] {
      DetectWallCollisionKernel(radius, (float4*)particle_pos4, (int*)rb_idx, (float4*)rb_vel4,
                                wall_pos, nrm, cn.data(), cp.data(), cw.data(), cd.data(), n);
    });
  }
  // particleIndices sorted by distance; body flags sorted by distance; then indices
  // sorted by flag (all stable).
  std::vector<uint32_t> key(n), ids(n), flags(n);
  long t = 0;
  for (int b = 0; b < num_bodies; ++b)
    for (int k = 0; k < particles_per_rb[b]; ++k) flags[t++] = (uint32_t)b;
  for (int i = 0; i < n; ++i) { key[i] = float_key_bits(cd[i]); ids[i] = (uint32_t)i; }
  std::vector<uint32_t> key2 = key;
  stable_lsd(key.data(), ids.data(), n);
  stable_lsd(key2.data(), flags.data(), n);
  stable_lsd(flags.data(), ids.data(), n);
  std::vector<int> contact_id(ids.begin(), ids.end());
  std::vector<int> cum(num_bodies);
  int run = 0;
  for (int b = 0; b < num_bodies; ++b) { run += particles_per_rb[b]; cum[b] = run; }
  launch(num_bodies, 128, true, [&] {
    HandleWallCollisionKernelUnmapped(radius, (float4*)rb_pos4, (float4*)rb_vel4,
                                      (float4*)rb_ang4, nullptr, nullptr,
                                      (glm::mat3*)inv_inertia9, (float*)rb_mass, cn.data(),
                                      cw.data(), cp.data(), cd.data(), contact_id.data(),
                                      cum.data(), num_bodies);
  });
}

}  // extern "C"

// ---- the sequential-impulse host loops (ParticleSystem members) ---------------------------
// The reference's default update gathers one contact per colliding particle and solves them
// with a sequential-impulse loop on the host (Particles/updateFunctions.cpp:1431-1874).  Those
// are member functions of ParticleSystem working on host copies of its device arrays.  The
// stand-in class below holds exactly the members the extracted bodies use; every array it
// points to is host memory here, so the device<->host copies become memcpy.  The solver's
// tail call re-poses the particles with the computeGlobalAttributes kernel body, launched
// over the grid the reference wrapper uses (Kernels/rigidBodyKernels.cu:423-447).
#include <cstdlib>
using std::abs;  // the reference's MSVC build resolves abs(float) to the float overload

namespace {
cudaError_t host_copy(void* dst, const void* src, size_t bytes) {
  std::memcpy(dst, src, bytes);
  return cudaSuccess;
}
}  // namespace

void computeGlobalAttributesWrapper(float4* CMs, float4* rigidVel, float4* relativePos,
                                    float4* globalPos, float4* globalVel, glm::quat* rbQuaternion,
                                    float4* rbAngularVelocity, int* rigidBodyIndex,
                                    int numParticles, int numThreads) {
  launch(numParticles, numThreads, true, [&] {
    computeGlobalAttributes(CMs, rigidVel, relativePos, globalPos, globalVel, rbQuaternion,
                            rbAngularVelocity, rigidBodyIndex, numParticles);
  });
}

class ParticleSystem {
 public:
  SimParams m_params;
  int numRigidBodies = 0, m_numParticles = 0, numberOfRangeData = 0, numThreads = 128;
  int* particlesPerObjectThrown = nullptr;
  float4 *rbPositions = nullptr, *rbVelocities = nullptr, *rbAngularVelocity = nullptr;
  float4 *relativePos = nullptr, *dPos = nullptr, *m_dVel = nullptr;
  float4 *staticNorm = nullptr, *contact_normal = nullptr;
  glm::mat3* rbCurrentInertia = nullptr;
  float* rbMass = nullptr;
  glm::quat* rbQuaternion = nullptr;
  int* rbIndices = nullptr;
  float* contactDistance = nullptr;
  int *collidingRigidBodyIndex = nullptr, *collidingParticleIndex = nullptr;
  std::vector<float4> ContactNormal, ContactPoint;
  std::vector<int> ContactRigidBody_1, ContactRigidBody_2;
  std::vector<float> ContactAccumulatedImpulse, ContactAccumulatedFriction,
      ContactAccumulatedFriction_2, ContactBias;
  void findExactContactPoint(const float4& p1, const float4& p2, const float& r1,
                             const float& r2, float4& cp, float4& cn);
  void GatherRigidBodyCollisions();
  void GatherAugmentedRealityCollisions();
  void SequentialImpulseSolver();
};

#undef checkCudaErrors
#define checkCudaErrors(val) (val)
#define cudaMemcpy(dst, src, bytes, kind) host_copy((dst), (src), (bytes))
#define cudaGetLastError() cudaSuccess
#define cudaDeviceSynchronize() cudaSuccess
#include "extracted_members.inc"
#undef cudaMemcpy
#undef cudaGetLastError
#undef cudaDeviceSynchronize

extern "C" {

// One gather (GatherRigidBodyCollisions, or GatherAugmentedRealityCollisions when
// `static_scene` is set: then contact_body is unused and scene_normals4 gives the normals)
// followed, when iterations_run > 0, by SequentialImpulseSolver on the gathered contacts.
// Body state is updated in place (vel4, ang4); pos4 / pvel4 / quat4 receive the re-posed
// particles.  Writes up to `capacity` contacts (normal, point, body1, body2, bias and the three
// accumulated impulses after the solve) and returns the number gathered.
int refcpu_sis_step(const void* sim_params, int num_bodies, int n, const int* particles_per_rb,
                    float* cms4, float* vel4, float* ang4, float* inertia9, float* mass,
                    float* rel4, float* pos4, float* pvel4, float* quat4, int* rb_idx,
                    float* contact_distance, int* contact_body, int* contact_particle,
                    float* scene_normals4, int num_scene_points, int static_scene,
                    int solve, int capacity, float* out_normal4, float* out_point4,
                    int* out_body1, int* out_body2, float* out_bias, float* out_acc) {
  ParticleSystem ps;
  std::memcpy(&ps.m_params, sim_params, sizeof(SimParams));
  ps.numRigidBodies = num_bodies;
  ps.m_numParticles = n;
  ps.numberOfRangeData = num_scene_points;
  ps.particlesPerObjectThrown = const_cast<int*>(particles_per_rb);
  ps.rbPositions = (float4*)cms4;
  ps.rbVelocities = (float4*)vel4;
  ps.rbAngularVelocity = (float4*)ang4;
  ps.relativePos = (float4*)rel4;
  ps.dPos = (float4*)pos4;
  ps.m_dVel = (float4*)pvel4;
  ps.staticNorm = (float4*)scene_normals4;
  std::vector<float4> cn_scratch((size_t)n);
  ps.contact_normal = cn_scratch.data();
  ps.rbCurrentInertia = (glm::mat3*)inertia9;
  ps.rbMass = mass;
  ps.rbQuaternion = (glm::quat*)quat4;
  ps.rbIndices = rb_idx;
  ps.contactDistance = contact_distance;
  ps.collidingRigidBodyIndex = contact_body;
  ps.collidingParticleIndex = contact_particle;
  if (static_scene) ps.GatherAugmentedRealityCollisions();
  else ps.GatherRigidBodyCollisions();
  if (solve) ps.SequentialImpulseSolver();
  const int k = (int)ps.ContactNormal.size();
  for (int c = 0; c < k && c < capacity; ++c) {
    std::memcpy(out_normal4 + 4 * (size_t)c, &ps.ContactNormal[c], 16);
    std::memcpy(out_point4 + 4 * (size_t)c, &ps.ContactPoint[c], 16);
    out_body1[c] = ps.ContactRigidBody_1[c];
    out_body2[c] = ps.ContactRigidBody_2[c];
    out_bias[c] = ps.ContactBias[c];
    out_acc[3 * (size_t)c] = ps.ContactAccumulatedImpulse[c];
    out_acc[3 * (size_t)c + 1] = ps.ContactAccumulatedFriction[c];
    out_acc[3 * (size_t)c + 2] = ps.ContactAccumulatedFriction_2[c];
  }
  return k;
}

}  // extern "C"

// ---- particle-body files: the body set-up of ParticleSystem::initObject -------------------
// (RigidBodies/RigidBodyAddition.cpp:1576-1756, extracted into
// oracle/_ref/extracted_init_object.inc.)  The file's text is given as a string; the
// statements run with the locals they expect: the particle array m_hPos (4 floats per
// particle), the stream positioned after the count line, the model name, scale and particle
// radius, and a particle velocity array it zeroes.  Returns the particle count; writes the
// centred offsets and the inverse inertia
// (glm::mat3 memory order).
#include <sstream>
#include <string>

extern "C" int refcpu_init_object(const char* text, const char* modelName, float scale,
                                  float particle_radius, float* rel4, float* inv_inertia9) {
  std::istringstream myfile{std::string(text)};
  std::string line;
  std::getline(myfile, line);
  const int particles = std::atoi(line.c_str());
  const int start = 0;
  std::vector<float> h_pos(4 * (size_t)particles), h_vel(4 * (size_t)particles);
  float* m_hPos = h_pos.data();
  float* m_hVel = h_vel.data();
  struct {
    float particleRadius;
  } m_params{particle_radius};
  const bool initializedNow = true;
  int m_numParticles = 0;
#include "extracted_init_object.inc"
  (void)m_numParticles;
  std::memcpy(rel4, m_hPos, 4 * sizeof(float) * (size_t)particles);
  std::memcpy(inv_inertia9, &inertiaTensor[0][0], 9 * sizeof(float));
  return particles;
}

// ---- depth-camera ingestion: RGBDloader and computeNormals (Kernels/customRangeImageLoader.cu
// :14-177) over the grid loadRangeImage launches (:179-221): 16 x 32 blocks, width / 16 x
// height / 32 of them.  vao5 must hold 5 floats per pixel (the kernel writes it always).
namespace {
template <class F>
void launch_image(int w, int h, F&& body) {
  const int bx = 16, by = 32, gx = w / bx, gy = h / by;
  for (int yb = 0; yb < gy; ++yb)
    for (int xb = 0; xb < gx; ++xb)
      for (int ty = 0; ty < by; ++ty)
        for (int tx = 0; tx < bx; ++tx) {
          blockIdx = make_uint3((unsigned)xb, (unsigned)yb, 0);
          threadIdx = make_uint3((unsigned)tx, (unsigned)ty, 0);
          blockDim = dim3(bx, by, 1);
          gridDim = dim3(gx, gy, 1);
          body();
        }
}
}  // namespace

extern "C" void refcpu_range_cloud(const unsigned short* depth, int w, int h, const float* cam16,
                                   float radius, float* pos4, float* radii, float* vao5) {
  glm::mat4 cam;
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r) cam[c][r] = cam16[4 * c + r];
  launch_image(w, h, [&] {
    RGBDloader(const_cast<unsigned short*>(depth), vao5, pos4, cam, radii, radius, w, h);
  });
}

extern "C" void refcpu_range_normals(const float* pos4, int w, int h, float* norm4) {
  launch_image(w, h, [&] {
    computeNormals(reinterpret_cast<float4*>(const_cast<float*>(pos4)),
                   reinterpret_cast<float4*>(norm4), w, h);
  });
}
