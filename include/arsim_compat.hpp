/*
 * arsim_compat.hpp -- the reference's kernel-wrapper API, implemented on libarsim.so.
 *
 * AR_Sim's simulator host code (ParticleSystem, Particles/updateFunctions.cpp,
 * RigidBodies/UniformGridUpdate.cpp, RigidBodies/BVHUpdate.cpp) calls free C++ functions
 * declared in Particles/ParticleAuxiliaryFunctions.h, BVHSource/BVHcreation.h and
 * RigidBodies/rigidBodyKernelWrappers.h.  This header defines those functions with the same
 * names and signatures (C++ linkage; SimParams, AABB, float4 and glm types from the
 * project's own headers), each forwarding to the C ABI in arsim.h.  To switch a build over:
 *   1. drop the reference's .cu kernel files from the build;
 *   2. in exactly one .cpp, after the project headers that define SimParams, AABB and glm:
 *        #define ARSIM_COMPAT_IMPLEMENTATION
 *        #include "arsim_compat.hpp"
 *   3. link libarsim.so.
 *
 * Behaviour kept from the reference: the same array layouts, in-place updates and the
 * `**` buffer swaps of the sort wrappers (after a sort, *keys points at the sorted data and
 * the "sorted" pointer at the spare buffer, like cub::DoubleBuffer::Current/Alternate);
 * host-side `particlesPerObject` counts are uploaded per call.  Work runs on the legacy
 * default stream and each wrapper synchronises before returning, as the reference's
 * checkCudaErrors(cudaDeviceSynchronize()) calls do.  Differences, by design: no
 * allocation per call (a process-wide context owns the workspace); per-body sums are the
 * fixed-order segmented sums (the reference's prefix-sum differences drop each body's first
 * particle, UniformGridDEM.cu:440-441); BVH traversal needs no stack.
 *
 * Errors: the reference exits through checkCudaErrors.  Here a failing wrapper calls the
 * handler installed with arsim_compat_set_error_handler (default: print and exit(1)).
 */
#ifndef ARSIM_COMPAT_HPP
#define ARSIM_COMPAT_HPP

#include <cuda_runtime.h>

#include "arsim.h"

typedef void (*arsim_compat_error_handler)(ar_status status, const char* where,
                                           const char* message);
void arsim_compat_set_error_handler(arsim_compat_error_handler handler);
/* The process-wide context the wrappers use (created on the current device on first use). */
ar_ctx* arsim_compat_context();

#ifdef ARSIM_COMPAT_IMPLEMENTATION
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace arsim_compat_detail {

inline void default_handler(ar_status s, const char* where, const char* msg) {
  std::fprintf(stderr, "arsim: %s failed (status %d): %s\n", where, (int)s, msg);
  std::exit(EXIT_FAILURE);
}
static arsim_compat_error_handler g_handler = default_handler;
static ar_ctx* g_ctx = nullptr;
static SimParams g_params;  // setParameters target (the reference's __constant__ params)

inline void check(ar_status s, const char* where) {
  if (s == AR_OK) s = ar_ctx_status(g_ctx, nullptr);  // synchronise like the reference
  if (s != AR_OK) g_handler(s, where, ar_last_error());
}
inline const ar_sim_params* P(const SimParams& p) {
  static_assert(sizeof(SimParams) == sizeof(ar_sim_params), "SimParams layout differs");
  return reinterpret_cast<const ar_sim_params*>(&p);
}

// Device buffers for host-side per-body counts (grow-only).
struct DeviceInts {
  int32_t* ptr = nullptr;
  size_t cap = 0;
  int32_t* upload(const std::vector<int32_t>& v) {
    if (v.size() > cap) {
      if (ptr) cudaFree(ptr);
      cap = v.size() + 1024;
      if (cudaMalloc(&ptr, cap * sizeof(int32_t)) != cudaSuccess) {
        ptr = nullptr;
        cap = 0;
        return nullptr;
      }
    }
    cudaMemcpy(ptr, v.data(), v.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
    return ptr;
  }
};
static DeviceInts g_offsets, g_starts, g_counts;

// Grow-only device scratch (32-bit words) for wrappers that need temporaries.
struct DeviceWords {
  uint32_t* ptr = nullptr;
  size_t cap = 0;
  uint32_t* reserve(size_t n) {
    if (n > cap) {
      if (ptr) cudaFree(ptr);
      cap = n + n / 4 + 64;
      if (cudaMalloc(&ptr, cap * sizeof(uint32_t)) != cudaSuccess) {
        cudaGetLastError();
        ptr = nullptr;
        cap = 0;
      }
    }
    return ptr;
  }
};
static DeviceWords g_spare_keys, g_spare_vals, g_box;

inline std::vector<int32_t> prefix(const int* counts, int n) {
  std::vector<int32_t> off(n + 1, 0);
  for (int i = 0; i < n; ++i) off[i + 1] = off[i] + counts[i];
  return off;
}

}  // namespace arsim_compat_detail

void arsim_compat_set_error_handler(arsim_compat_error_handler h) {
  arsim_compat_detail::g_handler = h ? h : arsim_compat_detail::default_handler;
}

ar_ctx* arsim_compat_context() {
  using namespace arsim_compat_detail;
  if (!g_ctx) {
    int dev = 0;
    cudaGetDevice(&dev);
    ar_status s = ar_ctx_create(dev, &g_ctx);
    if (s != AR_OK) g_handler(s, "ar_ctx_create", ar_last_error());
  }
  return g_ctx;
}

#define ARC_CTX arsim_compat_context()
#define ARC_CHECK(expr, name) arsim_compat_detail::check((expr), name)

/* ---- Particles/ParticleAuxiliaryFunctions.h ------------------------------------------------ */
void setParameters(SimParams* hostParams) { arsim_compat_detail::g_params = *hostParams; }

void integrateSystem(float* pos, float* vel, float deltaTime, float3 minPos, float3 maxPos,
                     int* rigidBodyIndices, uint numParticles) {
  const float mn[3] = {minPos.x, minPos.y, minPos.z}, mx[3] = {maxPos.x, maxPos.y, maxPos.z};
  ARC_CHECK(ar_integrate_particles(ARC_CTX, arsim_compat_detail::P(arsim_compat_detail::g_params),
                                   deltaTime, pos, vel, rigidBodyIndices, (int)numParticles, mn,
                                   mx, nullptr),
            "integrateSystem");
}

void calcHash(uint* gridParticleHash, uint* gridParticleIndex, float* pos, int numParticles) {
  ARC_CHECK(ar_calc_hash(ARC_CTX, arsim_compat_detail::P(arsim_compat_detail::g_params), pos,
                         numParticles, gridParticleHash, gridParticleIndex, nullptr),
            "calcHash");
}

void reorderDataAndFindCellStart(int* rbIndices, uint* cellStart, uint* cellEnd, float* sortedPos,
                                 float* sortedVel, uint* gridParticleHash,
                                 uint* gridParticleIndex, float* oldPos, float* oldVel,
                                 uint numParticles, uint numCells) {
  (void)rbIndices;
  ARC_CHECK(ar_reorder_cells(ARC_CTX, gridParticleHash, gridParticleIndex, oldPos, oldVel,
                             (int)numParticles, numCells, cellStart, cellEnd, sortedPos,
                             sortedVel, nullptr),
            "reorderDataAndFindCellStart");
}

void collide(float4* pForce, int* rbIndices, float4* relativePos, float4* pTorque, float* color,
             float* newVel, float* sortedPos, float* sortedVel, uint* gridParticleIndex,
             uint* cellStart, uint* cellEnd, uint numParticles, uint numCells) {
  (void)color;
  (void)numCells;
  ARC_CHECK(ar_collide_grid_particles(ARC_CTX,
                                      arsim_compat_detail::P(arsim_compat_detail::g_params),
                                      rbIndices, sortedPos, sortedVel, (float*)relativePos,
                                      gridParticleIndex, cellStart, cellEnd, (int)numParticles,
                                      (float*)pForce, (float*)pTorque, newVel, nullptr),
            "collide");
}

void sortParticlesPreallocated(uint** dGridParticleHash, uint** dGridParticleIndex,
                               uint** sortedGridParticleHash, uint** sortedGridParticleIndex,
                               uint numParticles) {
  ARC_CHECK(ar_radix_sort_pairs_u32(ARC_CTX, *dGridParticleHash, *dGridParticleIndex,
                                    *sortedGridParticleHash, *sortedGridParticleIndex,
                                    (int)numParticles, 0, 32, nullptr),
            "sortParticlesPreallocated");
  uint* k = *dGridParticleHash;
  uint* v = *dGridParticleIndex;
  *dGridParticleHash = *sortedGridParticleHash;   // Current()
  *dGridParticleIndex = *sortedGridParticleIndex;
  *sortedGridParticleHash = k;                    // Alternate()
  *sortedGridParticleIndex = v;
}

void sortParticles(uint** dGridParticleHash, uint** dGridParticleIndex, uint numParticles) {
  // sorted in place, through a spare pair of buffers that grows only when a call sorts more
  // pairs than any call before it (no allocation per call in steady state)
  using arsim_compat_detail::g_spare_keys;
  using arsim_compat_detail::g_spare_vals;
  uint32_t* k2 = g_spare_keys.reserve(numParticles);
  uint32_t* v2 = g_spare_vals.reserve(numParticles);
  if (!k2 || !v2) {
    arsim_compat_detail::g_handler(AR_ERR_OOM, "sortParticles", "spare sort buffers");
    return;
  }
  ARC_CHECK(ar_radix_sort_pairs_u32(ARC_CTX, *dGridParticleHash, *dGridParticleIndex, k2, v2,
                                    (int)numParticles, 0, 32, nullptr),
            "sortParticles");
  cudaMemcpy(*dGridParticleHash, k2, sizeof(uint) * numParticles, cudaMemcpyDeviceToDevice);
  cudaMemcpy(*dGridParticleIndex, v2, sizeof(uint) * numParticles, cudaMemcpyDeviceToDevice);
}

void createMortonCodesPreallocated(float4* positions, unsigned int** mortonCodes, int** indices,
                                   unsigned int** sortedMortonCodes, int** sortedIndices,
                                   float4 minPos, float4 maxPos, int elements,
                                   int numberOfThreads) {
  (void)numberOfThreads;
  const float mn[4] = {minPos.x, minPos.y, minPos.z, minPos.w};
  const float mx[4] = {maxPos.x, maxPos.y, maxPos.z, maxPos.w};
  ARC_CHECK(ar_morton30_box(ARC_CTX, (float*)positions, elements, mn, mx, *mortonCodes, *indices,
                            nullptr),
            "createMortonCodesPreallocated");
  ARC_CHECK(ar_radix_sort_pairs_u32(ARC_CTX, *mortonCodes, (uint32_t*)*indices,
                                    *sortedMortonCodes, (uint32_t*)*sortedIndices, elements, 0, 32,
                                    nullptr),
            "createMortonCodesPreallocated");
  // after the sort *sorted* hold the result (Current) and the inputs are the spare buffers
}

void initializeRadiiWrapper(float* radii, float particleRadius, int numParticles, int numThreads) {
  (void)numThreads;
  ARC_CHECK(ar_fill_f32(ARC_CTX, radii, numParticles, particleRadius, nullptr),
            "initializeRadiiWrapper");
}

/* ---- BVHSource/BVHcreation.h ----------------------------------------------------------------- */
cudaError_t createMortonCodes(float4* positions, unsigned int** mortonCodes, int** indices,
                              unsigned int** sortedMortonCodes, int** sortedIndices,
                              int numberOfPrimitives, int numberOfThreads) {
  (void)numberOfThreads;
  // the scene box (min, max) lives in a buffer allocated on the first call only
  float4* box = reinterpret_cast<float4*>(arsim_compat_detail::g_box.reserve(8));
  if (!box) return cudaErrorMemoryAllocation;
  ar_status s = ar_scene_aabb(ARC_CTX, (float*)positions, numberOfPrimitives, (float*)box,
                              (float*)(box + 1), nullptr);
  if (s == AR_OK)
    s = ar_morton30(ARC_CTX, (float*)positions, numberOfPrimitives, (float*)box,
                    (float*)(box + 1), *mortonCodes, *indices, nullptr);
  if (s == AR_OK)
    s = ar_radix_sort_pairs_u32(ARC_CTX, *mortonCodes, (uint32_t*)*indices, *sortedMortonCodes,
                                (uint32_t*)*sortedIndices, numberOfPrimitives, 0, 32, nullptr);
  if (s == AR_OK) s = ar_ctx_status(ARC_CTX, nullptr);
  return s == AR_OK ? cudaSuccess : cudaErrorUnknown;
}

void wrapperConstructRadixTreeSoA(bool* isLeaf, int* leftIndices, int* rightIndices,
                                  int* parentIndices, int* minRange, int* maxRange,
                                  unsigned int* sortedMortonCodes, int numThreads,
                                  int numParticles) {
  (void)numThreads;
  ARC_CHECK(ar_lbvh_build(ARC_CTX, sortedMortonCodes, numParticles, (uint8_t*)isLeaf,
                          leftIndices, rightIndices, parentIndices, minRange, maxRange, nullptr),
            "wrapperConstructRadixTreeSoA");
}

void wrapperConstructLeafNodesSoA(bool* isLeaf, int* leftIndices, int* rightIndices,
                                  int* parentIndices, int* minRange, int* maxRange, float4* CMs,
                                  AABB* bounds, int* sortedIndices, float* radii,
                                  float4* positions, float particleRadius, int numThreads,
                                  int numParticles) {
  (void)leftIndices;
  (void)rightIndices;
  (void)parentIndices;
  (void)numThreads;
  ARC_CHECK(ar_lbvh_leaves(ARC_CTX, numParticles, sortedIndices, (float*)positions,
                           particleRadius, (uint8_t*)isLeaf, minRange, maxRange, (float*)CMs,
                           (float*)bounds, radii, nullptr),
            "wrapperConstructLeafNodesSoA");
}

void wrapperConstructInternalNodesSoA(int* leftIndices, int* rightIndices, int* parentIndices,
                                      AABB* bounds, int numThreads, int numParticles) {
  (void)numThreads;
  ARC_CHECK(ar_lbvh_refit(ARC_CTX, numParticles, leftIndices, rightIndices, parentIndices,
                          (float*)bounds, nullptr),
            "wrapperConstructInternalNodesSoA");
}

/* ---- RigidBodies/rigidBodyKernelWrappers.h ----------------------------------------------------- */
void integrateSystemRigidBodies(float4* CMs, float4* vel, float4* force, float4* rbAngularVelocity,
                                glm::quat* rbQuaternion, float4* rbTorque,
                                float4* rbAngularMomentum, float4* rbLinearMomentum,
                                glm::mat3* rbInertia, glm::mat3* rbCurrentInertia,
                                glm::vec3* rbAngularAcceleration, float deltaTime, float* rbRadii,
                                float* rbMass, float3 minPos, float3 maxPos, int numBodies,
                                SimParams params, int numThreads) {
  (void)numThreads;
  const float mn[3] = {minPos.x, minPos.y, minPos.z}, mx[3] = {maxPos.x, maxPos.y, maxPos.z};
  ARC_CHECK(ar_integrate_momentum(ARC_CTX, arsim_compat_detail::P(params), deltaTime, numBodies,
                                  (float*)CMs, (float*)vel, (float*)force,
                                  (float*)rbAngularVelocity, (float*)rbQuaternion,
                                  (float*)rbTorque, (float*)rbAngularMomentum,
                                  (float*)rbLinearMomentum, (const float*)rbInertia,
                                  (float*)rbCurrentInertia, (float*)rbAngularAcceleration,
                                  rbRadii, rbMass, mn, mx, nullptr),
            "integrateSystemRigidBodies");
}

void GPUintegratorWrapper(float4* CMs, float4* vel, float4* rbAngularVelocity,
                          glm::quat* rbQuaternion, glm::mat3* rbInertia,
                          glm::mat3* rbCurrentInertia, glm::mat4* modelMatrixGPU,
                          glm::quat* cumulativeQuaternionGPU, float deltaTime, float* rbMass,
                          int numBodies, SimParams params, int numThreads) {
  (void)numThreads;
  ARC_CHECK(ar_integrate_reference(ARC_CTX, arsim_compat_detail::P(params), deltaTime, numBodies,
                                   (float*)CMs, (float*)vel, (float*)rbAngularVelocity,
                                   (float*)rbQuaternion, (const float*)rbInertia,
                                   (float*)rbCurrentInertia, (float*)modelMatrixGPU,
                                   (float*)cumulativeQuaternionGPU, rbMass, nullptr),
            "GPUintegratorWrapper");
}

void computeGlobalAttributesWrapper(float4* CMs, float4* rigidVel, float4* relativePos,
                                    float4* globalPos, float4* globalVel,
                                    glm::quat* rbQuaternion, float4* rbAngularVelocity,
                                    int* rigidBodyIndex, int numParticles, int numThreads) {
  (void)numThreads;
  ARC_CHECK(ar_global_attributes(ARC_CTX, numParticles, 0, (float*)CMs, (float*)rigidVel,
                                 (float*)rbAngularVelocity, (float*)rbQuaternion, rigidBodyIndex,
                                 (float*)relativePos, (float*)globalPos, (float*)globalVel,
                                 nullptr),
            "computeGlobalAttributesWrapper");
}

void resetQuaternionWrapper(glm::quat* rbQuaternion, int numRigidBodies, int numThreads) {
  (void)numThreads;
  ARC_CHECK(ar_reset_quaternions(ARC_CTX, (float*)rbQuaternion, numRigidBodies, nullptr),
            "resetQuaternionWrapper");
}

void ResetParticleImpulseWrapper(float4* pLinearImpulse, float4* pAngularImpulse,
                                 int numParticles, int numThreads) {
  (void)numThreads;
  ARC_CHECK(ar_fill_f32(ARC_CTX, (float*)pLinearImpulse, 4l * numParticles, 0.f, nullptr),
            "ResetParticleImpulseWrapper");
  ARC_CHECK(ar_fill_f32(ARC_CTX, (float*)pAngularImpulse, 4l * numParticles, 0.f, nullptr),
            "ResetParticleImpulseWrapper");
}

void FindAndHandleRigidBodyCollisionsUniformGridWrapper(
    int* rbIndices, float4* pLinearImpulse, float4* pAngularImpulse, float4* color,
    float4* sortedPos, float4* sortedVel, float4* relativePos, float3 minPos, float3 maxPos,
    uint* gridParticleIndex, uint* cellStart, uint* cellEnd, uint numParticles,
    SimParams params, int numThreads) {
  (void)color;
  (void)minPos;
  (void)maxPos;
  (void)numThreads;
  ARC_CHECK(ar_collide_grid_dem(ARC_CTX, arsim_compat_detail::P(params), rbIndices,
                                (float*)sortedPos, (float*)sortedVel, (float*)relativePos,
                                gridParticleIndex, cellStart, cellEnd, (int)numParticles,
                                (float*)pLinearImpulse, (float*)pAngularImpulse, nullptr),
            "FindAndHandleRigidBodyCollisionsUniformGridWrapper");
}

void FindAndHandleAugmentedRealityCollisionsUniformGridWrapper(
    float4* pLinearImpulse, float4* pAngularImpulse, float4* color, float4* sortedPos,
    float4* sortedVel, float4* relativePos, float4* ARPos, float4* ARnormals,
    uint* gridParticleIndex, uint* gridParticleIndexAR, uint* cellStart, uint* cellEnd,
    uint numParticles, SimParams params, int numThreads) {
  (void)numThreads;
  ARC_CHECK(ar_collide_static_scene_dem(
                ARC_CTX, arsim_compat_detail::P(params), (float*)sortedPos, (float*)sortedVel,
                (float*)relativePos, (float*)ARPos, (float*)ARnormals, gridParticleIndex,
                gridParticleIndexAR, cellStart, cellEnd, (int)numParticles,
                (float*)pLinearImpulse, (float*)pAngularImpulse, (float*)color, nullptr),
            "FindAndHandleAugmentedRealityCollisionsUniformGridWrapper");
}

// FindRigidBodyCollisionsUniformGridWrapper (Kernels/RB_UniformGridKernels.cu:844-874): the
// deepest contact per particle.  The reference's debug colouring of colliding particles
// (color) is not written.
void FindRigidBodyCollisionsUniformGridWrapper(int* rbIndices, int* collidingRigidBodyIndex,
                                               int* collidingParticleIndex,
                                               float* contactDistance, float4* color,
                                               float4* oldPos, uint* gridParticleIndex,
                                               uint* cellStart, uint* cellEnd,
                                               uint numParticles, SimParams params,
                                               int numThreads) {
  (void)color;
  (void)numThreads;
  ARC_CHECK(ar_find_contacts_grid(ARC_CTX, arsim_compat_detail::P(params), rbIndices,
                                  (const float*)oldPos, gridParticleIndex, cellStart, cellEnd,
                                  (int)numParticles, contactDistance, collidingRigidBodyIndex,
                                  collidingParticleIndex, nullptr),
            "FindRigidBodyCollisionsUniformGridWrapper");
}

void ReducePerParticleImpulses(int* rbIndices, float4* pLinearImpulse, float4* pAngularImpulse,
                               float4* rbVel, float4* rbAng, float* rbMass, glm::mat3* rbInertia,
                               int* particlesPerObject, int numRigidBodies, int numParticles,
                               int numThreads) {
  (void)rbIndices;
  (void)numParticles;
  (void)numThreads;
  int32_t* off = arsim_compat_detail::g_offsets.upload(
      arsim_compat_detail::prefix(particlesPerObject, numRigidBodies));
  ARC_CHECK(off ? ar_reduce_impulses(ARC_CTX, (float*)pLinearImpulse, (float*)pAngularImpulse,
                                     off, numRigidBodies, (float*)rbVel, (float*)rbAng, rbMass,
                                     (const float*)rbInertia, nullptr)
                : AR_ERR_OOM,
            "ReducePerParticleImpulses");
}

void ReduceRigidBodyVariables(float4* rbForce, float4* rbTorque, float4* rbPositions,
                              float4* pForce, float4* pTorque, float4* pPositions,
                              int* particlesPerObjectThrown, bool* isRigidBody, int objectsThrown,
                              int numRigidBodies, int numThreads, int numParticles,
                              bool* toExit) {
  (void)rbPositions;
  (void)pPositions;
  (void)numThreads;
  (void)numParticles;
  std::vector<int32_t> starts, counts;
  int run = 0;
  for (int o = 0; o < objectsThrown; ++o) {
    if (isRigidBody[o]) {
      starts.push_back(run);
      counts.push_back(particlesPerObjectThrown[o]);
    }
    run += particlesPerObjectThrown[o];
  }
  (void)numRigidBodies;
  int32_t* ds = arsim_compat_detail::g_starts.upload(starts);
  int32_t* dc = arsim_compat_detail::g_counts.upload(counts);
  ar_status s = (ds && dc) ? ar_reduce_rigid_body_variables(ARC_CTX, (float*)pForce,
                                                            (float*)pTorque, ds, dc,
                                                            (int)starts.size(), (float*)rbForce,
                                                            (float*)rbTorque, nullptr)
                           : AR_ERR_OOM;
  if (s == AR_OK) s = ar_ctx_status(ARC_CTX, nullptr);
  if (s == AR_ERR_NAN) {
    if (toExit) *toExit = true;  // the reference flags NaN sums this way
    return;
  }
  ARC_CHECK(s, "ReduceRigidBodyVariables");
}

void WallCollisionWrapper(float4* particlePos, float4* rbPos, float3 minPos, float3 maxPos,
                          float4* rbVel, float4* rbAng, float4* rbLinMom, float4* rbAngMom,
                          glm::mat3* Iinv, float* rbMass, int* rbIndices, int* particlesPerRB,
                          int numRigidBodies, int numParticles, int numThreads,
                          SimParams params) {
  (void)rbLinMom;
  (void)rbAngMom;
  (void)numThreads;
  const float mn[3] = {minPos.x, minPos.y, minPos.z}, mx[3] = {maxPos.x, maxPos.y, maxPos.z};
  int32_t* off = arsim_compat_detail::g_offsets.upload(
      arsim_compat_detail::prefix(particlesPerRB, numRigidBodies));
  ARC_CHECK(off ? ar_walls_reference(ARC_CTX, params.particleRadius, (float*)particlePos,
                                     (float*)rbPos, mn, mx, (float*)rbVel, (float*)rbAng,
                                     (const float*)Iinv, rbMass, rbIndices, off, numRigidBodies,
                                     numParticles, nullptr)
                : AR_ERR_OOM,
            "WallCollisionWrapper");
}

void collideBVHSoARigidBodyWrapper(float4* color, float4* pForce, int* rigidBodyIndex,
                                   float4* pPositions, float4* positions, float4* relativePos,
                                   float4* pTorque, float4* vel, bool* isLeaf, int* leftIndices,
                                   int* rightIndices, int* minRange, int* maxRange, float4* CMs,
                                   AABB* bounds, int* sortedIndices, float* radii,
                                   int numParticles, int numThreads, SimParams params) {
  (void)color;
  (void)positions;
  (void)minRange;
  (void)maxRange;
  (void)numThreads;
  ARC_CHECK(ar_collide_bvh_dem(ARC_CTX, arsim_compat_detail::P(params), rigidBodyIndex,
                               (float*)relativePos, (float*)vel, (uint8_t*)isLeaf, leftIndices,
                               rightIndices, nullptr, (float*)CMs, (float*)bounds, sortedIndices,
                               radii, numParticles, (float*)pForce, (float*)pTorque,
                               (float*)pPositions, nullptr),
            "collideBVHSoARigidBodyWrapper");
}

void FindRigidBodyCollisionsBVHWrapper(float4* color, int* rigidBodyIndex, bool* isLeaf,
                                       int* leftIndices, int* rightIndices, int* minRange,
                                       int* maxRange, float4* CMs, AABB* bounds,
                                       int* sortedIndices, float* radii, int numThreads,
                                       int numParticles, SimParams params,
                                       float* contactDistance, int* collidingParticleIndex,
                                       int* collidingRigidBodyIndex) {
  (void)color;
  (void)minRange;
  (void)numThreads;
  (void)params;
  ARC_CHECK(ar_find_contacts_bvh(ARC_CTX, rigidBodyIndex, (uint8_t*)isLeaf, leftIndices,
                                 rightIndices, nullptr, maxRange, (float*)CMs, (float*)bounds,
                                 sortedIndices, radii, numParticles, contactDistance,
                                 collidingParticleIndex, collidingRigidBodyIndex, nullptr),
            "FindRigidBodyCollisionsBVHWrapper");
}

/* ---- depth-camera ingestion: declared in Particles/loadRangeDataFromFile.cpp:13-22, defined in
 * Kernels/customRangeImageLoader.cu:179-221 (VAOdata: the mapped GL buffer there, any device
 * buffer of 5 floats per pixel here) ------------------------------------------------------- */
cudaError_t loadRangeImage(unsigned short* image, float** VAOdata, float** staticPos,
                           float** staticNorm, glm::mat4& cameraTransformation,
                           float* staticRadii, float particleRadius, int imageWidth,
                           int imageHeight) {
  float cam[16];
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r) cam[4 * c + r] = cameraTransformation[c][r];
  ARC_CHECK(ar_range_image_cloud(ARC_CTX, image, imageWidth, imageHeight, cam, particleRadius,
                                 *staticPos, staticRadii, *VAOdata, nullptr),
            "loadRangeImage");
  ARC_CHECK(ar_range_image_normals(ARC_CTX, *staticPos, imageWidth, imageHeight, *staticNorm,
                                   nullptr),
            "loadRangeImage");
  return cudaDeviceSynchronize();
}

#undef ARC_CTX
#undef ARC_CHECK
#endif /* ARSIM_COMPAT_IMPLEMENTATION */
#endif /* ARSIM_COMPAT_HPP */
