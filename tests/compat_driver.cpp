// Test driver for include/arsim_compat.hpp, the C++ shim with the reference's wrapper
// signatures.  It is compiled against the reference's own declaration headers (SimParams,
// AABB, float4, glm) and linked against libarsim.so, then called from Python with plain
// pointers, so that the GPU tests run each wrapper exactly as reference host code would:
// through its C++ signature, with its `**` buffer swaps, its host-side per-body counts and its
// by-value SimParams.  Every wrapper synchronises before it returns, like the reference's.
// Errors go to a handler that records the status instead of exiting the test process.
#define GLM_FORCE_CUDA
#include <glm/glm.hpp>
#include <glm/gtc/quaternion.hpp>

#include "ParticleAuxiliaryFunctions.h"
#include "rigidBodyKernelWrappers.h"
#define ARSIM_COMPAT_IMPLEMENTATION
#include "arsim_compat.hpp"

#include <cstring>

namespace {
int g_status = 0;
void record(ar_status s, const char*, const char*) {
  if (g_status == 0) g_status = (int)s;
}
SimParams params_of(const void* p) {
  SimParams s;
  std::memcpy(&s, p, sizeof(SimParams));
  return s;
}
float3 f3(const float* v) { return make_float3(v[0], v[1], v[2]); }
}  // namespace

extern "C" {

// Installs the recording error handler and creates the shim's context on the current device.
int drv_init() {
  arsim_compat_set_error_handler(record);
  g_status = 0;
  return arsim_compat_context() ? 0 : -1;
}

// First failure status since the last call (0 = none), then cleared.
int drv_take_status() {
  const int s = g_status;
  g_status = 0;
  return s;
}

int drv_sizeof_simparams() { return (int)sizeof(SimParams); }

void drv_set_params(const void* params) {
  SimParams p = params_of(params);
  setParameters(&p);
}

// sortParticlesPreallocated; out[0..3] = the four pointers afterwards (hash, index, sorted
// hash, sorted index), so the caller can check the swap.
void drv_sort_preallocated(uint32_t* hash, uint32_t* index, uint32_t* shash, uint32_t* sindex,
                           uint32_t n, void** out) {
  uint* h = hash;
  uint* i = index;
  uint* sh = shash;
  uint* si = sindex;
  sortParticlesPreallocated(&h, &i, &sh, &si, n);
  out[0] = h;
  out[1] = i;
  out[2] = sh;
  out[3] = si;
}

// sortParticles (in place); out[0..1] = the two pointers afterwards.
void drv_sort_in_place(uint32_t* hash, uint32_t* index, uint32_t n, void** out) {
  uint* h = hash;
  uint* i = index;
  sortParticles(&h, &i, n);
  out[0] = h;
  out[1] = i;
}

void drv_calc_hash(uint32_t* hash, uint32_t* index, float* pos, int n) {
  calcHash(hash, index, pos, n);
}

void drv_reorder(uint32_t* cell_start, uint32_t* cell_end, float* spos, float* svel,
                 uint32_t* shash, uint32_t* sindex, float* pos, float* vel, uint32_t n,
                 uint32_t ncell) {
  reorderDataAndFindCellStart(nullptr, cell_start, cell_end, spos, svel, shash, sindex, pos, vel,
                              n, ncell);
}

void drv_collide_grid_dem(const void* params, int* rb, float* pforce, float* ptorque,
                          float* spos, float* svel, float* rel, uint32_t* sindex,
                          uint32_t* cell_start, uint32_t* cell_end, uint32_t n) {
  FindAndHandleRigidBodyCollisionsUniformGridWrapper(
      rb, (float4*)pforce, (float4*)ptorque, nullptr, (float4*)spos, (float4*)svel,
      (float4*)rel, make_float3(0.f, 0.f, 0.f), make_float3(1.f, 1.f, 1.f), sindex, cell_start,
      cell_end, n, params_of(params), 128);
}

// ReducePerParticleImpulses with the per-body particle counts on the host, as the reference
// keeps them (particlesPerObject).
void drv_reduce_impulses(int* rb, float* pforce, float* ptorque, float* bvel, float* bang,
                         float* mass, float* inv_inertia, int* counts_host, int nb, int n) {
  ReducePerParticleImpulses(rb, (float4*)pforce, (float4*)ptorque, (float4*)bvel, (float4*)bang,
                            mass, (glm::mat3*)inv_inertia, counts_host, nb, n, 128);
}

void drv_walls(const void* params, float* ppos, float* bpos, const float* mn, const float* mx,
               float* bvel, float* bang, float* inv_inertia, float* mass, int* rb,
               int* counts_host, int nb, int n) {
  WallCollisionWrapper((float4*)ppos, (float4*)bpos, f3(mn), f3(mx), (float4*)bvel,
                       (float4*)bang, nullptr, nullptr, (glm::mat3*)inv_inertia, mass, rb,
                       counts_host, nb, n, 128, params_of(params));
}

// loadRangeImage with the camera as a glm::mat4 (column-major 16 floats in).
int drv_range_image(unsigned short* depth, float* vao5, float* pos4, float* norm4, float* radii,
                    const float* cam16, float radius, int w, int h) {
  glm::mat4 cam;
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r) cam[c][r] = cam16[4 * c + r];
  return (int)loadRangeImage(depth, &vao5, &pos4, &norm4, cam, radii, radius, w, h);
}

}  // extern "C"
