// BASELINE INFRASTRUCTURE ONLY: the reference's own GPU step (ParticleSystem::
// updateUniformGridDEM, RigidBodies/UniformGridUpdate.cpp:939-999) on this GPU.  The product
// never loads what this file builds.
//
// oracle/ref_gpu_build.py compiles the reference's CUDA sources where they lie --
// Kernels/particleKernels.cu, Kernels/rigidBodyKernels.cu, RigidBodies/UniformGridDEM.cu -- for
// sm_100a and links them with this host driver into oracle/_ref/libref_gpu.so.  The step runs
// the reference's own wrappers (GPUintegratorWrapper, computeGlobalAttributesWrapper,
// resetQuaternionWrapper, FindAndHandleRigidBodyCollisionsUniformGridWrapper,
// ReducePerParticleImpulses) with their per-call allocations and synchronisations, in the
// order of the reference's driver.  Kernels/particleKernelWrappers.cu does not compile with
// this toolkit (a goto over initialisations), so its three launches on this path -- calcHash,
// sortParticlesPreallocated and reorderDataAndFindCellStart
// (Kernels/particleKernelWrappers.cu:195-254, 419-534) -- are made here the way that file makes
// them: 512-thread blocks for the hash and the reorder, a full-grid cellStart memset, and
// cub::DeviceRadixSort::SortPairs over all 32 key bits with a per-call temporary allocation
// (CUB from this toolkit; the vendored Libs/cub is a 2016 snapshot).
//
// CUDA events between the stages give each stage's time on the GPU timeline, host work that
// keeps the GPU idle included (the wrappers allocate, copy and synchronise).
#include <chrono>
#include <cstring>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>
#define GLM_FORCE_CUDA
#include <glm/glm.hpp>
#include <glm/gtc/quaternion.hpp>

#include "ParticleAuxiliaryFunctions.h"
#include "rigidBodyKernelWrappers.h"

// Kernels of Kernels/particleKernels.cu launched by this driver.
__global__ void calcHashD(uint* gridParticleHash, uint* gridParticleIndex, float4* pos,
                          uint numParticles);
__global__ void reorderDataAndFindCellStartD(int* rbIndices, uint* cellStart, uint* cellEnd,
                                             float4* sortedPos, float4* sortedVel,
                                             uint* gridParticleHash, uint* gridParticleIndex,
                                             float4* oldPos, float4* oldVel, uint numParticles);

namespace {

constexpr int kStages = 7;  // integrate | reset | hash | sort | reorder | collide | reduce
constexpr int kThreads = 128;  // ParticleSystem's numThreads (Particles/particleSystem.cpp:45)

struct State {
  int n = 0, nb = 0;
  uint ncell = 0;
  float dt = 0.f;
  SimParams prm;
  float4 *rb_pos = nullptr, *rb_vel = nullptr, *rb_ang = nullptr;
  glm::quat* rb_quat = nullptr;
  glm::mat3 *rb_inertia = nullptr, *rb_cur_inertia = nullptr;
  float* rb_mass = nullptr;
  float4 *rel = nullptr, *pos = nullptr, *vel = nullptr, *p_force = nullptr,
         *p_torque = nullptr, *color = nullptr, *spos = nullptr, *svel = nullptr;
  int* rb_index = nullptr;
  uint *hash = nullptr, *index = nullptr, *shash = nullptr, *sindex = nullptr;
  uint *cell_start = nullptr, *cell_end = nullptr;
  std::vector<int> per_body;
  std::vector<glm::quat> cum_quat;
  std::vector<glm::mat4> model;
  cudaEvent_t ev[kStages + 1] = {};
};
State g;
char g_err[256] = "";

bool ok(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  std::snprintf(g_err, sizeof(g_err), "%s: %s", what, cudaGetErrorString(e));
  return false;
}

template <class T>
bool dev(T** p, size_t count) {
  return ok(cudaMalloc((void**)p, count * sizeof(T)), "cudaMalloc");
}

void compute_grid_size(uint n, uint block, uint& blocks, uint& threads) {
  threads = block < n ? block : n;
  blocks = (n + threads - 1) / threads;
}

// The three launches of Kernels/particleKernelWrappers.cu on this path.
void calc_hash() {
  uint blocks, threads;
  compute_grid_size((uint)g.n, 512, blocks, threads);
  calcHashD<<<blocks, threads>>>(g.hash, g.index, g.pos, (uint)g.n);
}

bool sort_pairs() {
  cub::DoubleBuffer<uint> keys(g.hash, g.shash), vals(g.index, g.sindex);
  size_t bytes = 0;
  void* tmp = nullptr;
  if (!ok(cub::DeviceRadixSort::SortPairs(tmp, bytes, keys, vals, g.n), "SortPairs size"))
    return false;
  if (!ok(cudaMalloc(&tmp, bytes), "sort temporary")) return false;
  const bool r = ok(cub::DeviceRadixSort::SortPairs(tmp, bytes, keys, vals, g.n), "SortPairs") &&
                 ok(cudaDeviceSynchronize(), "sort");
  cudaFree(tmp);
  // the `**` swap of sortParticlesPreallocated: the sorted buffers become the step's arrays
  g.hash = keys.Current();
  g.shash = keys.Alternate();
  g.index = vals.Current();
  g.sindex = vals.Alternate();
  return r;
}

void reorder() {
  uint blocks, threads;
  compute_grid_size((uint)g.n, 512, blocks, threads);
  cudaMemset(g.cell_start, 0xff, (size_t)g.ncell * sizeof(uint));
  const uint smem = sizeof(uint) * (threads + 1);
  reorderDataAndFindCellStartD<<<blocks, threads, smem>>>(g.rb_index, g.cell_start, g.cell_end,
                                                        g.spos, g.svel, g.hash, g.index, g.pos,
                                                        g.vel, (uint)g.n);
}

void release() {
  void* ptrs[] = {g.rb_pos, g.rb_vel, g.rb_ang, g.rb_quat, g.rb_inertia, g.rb_cur_inertia,
                  g.rb_mass, g.rel, g.pos, g.vel, g.p_force, g.p_torque, g.color, g.spos,
                  g.svel, g.rb_index, g.hash, g.index, g.shash, g.sindex, g.cell_start,
                  g.cell_end};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (cudaEvent_t& e : g.ev)
    if (e) cudaEventDestroy(e);
  g = State();
}

}  // namespace

extern "C" {

const char* ref_gpu_last_error() { return g_err; }
int ref_gpu_stages() { return kStages; }

// Uploads a scene in the reference's layout: body centre, velocity and angular velocity as
// float4, orientation as glm::quat (x, y, z, w) -- the per-step quaternion starts at the
// identity and the cumulative one at `cum_quat4` --, inverse inertia (glm::mat3), mass, the
// particles' world-frame offsets and body indices, particles per body; `params` is the
// reference's SimParams (128 bytes).  Returns 0 on success.
int ref_gpu_create(int n, int nb, const float* body_pos4, const float* body_vel4,
                   const float* body_ang4, const float* cum_quat4, const float* inv_inertia9,
                   const float* mass, const float* rel4, const int* rb_index,
                   const int* per_body, const void* params, float dt) {
  release();
  g.n = n;
  g.nb = nb;
  g.dt = dt;
  std::memcpy(&g.prm, params, sizeof(SimParams));
  g.ncell = g.prm.numCells;
  const bool a = dev(&g.rb_pos, nb) && dev(&g.rb_vel, nb) && dev(&g.rb_ang, nb) &&
                 dev(&g.rb_quat, nb) && dev(&g.rb_inertia, nb) && dev(&g.rb_cur_inertia, nb) &&
                 dev(&g.rb_mass, nb) && dev(&g.rel, n) && dev(&g.pos, n) && dev(&g.vel, n) &&
                 dev(&g.p_force, n) && dev(&g.p_torque, n) && dev(&g.color, n) &&
                 dev(&g.spos, n) && dev(&g.svel, n) && dev(&g.rb_index, n) && dev(&g.hash, n) &&
                 dev(&g.index, n) && dev(&g.shash, n) && dev(&g.sindex, n) &&
                 dev(&g.cell_start, g.ncell) && dev(&g.cell_end, g.ncell);
  if (!a) {
    release();
    return 1;
  }
  std::vector<glm::quat> ident(nb, glm::quat(1.f, 0.f, 0.f, 0.f));
  g.cum_quat.resize(nb);
  std::memcpy(g.cum_quat.data(), cum_quat4, sizeof(float) * 4 * nb);
  g.model.assign(nb, glm::mat4(1.f));
  g.per_body.assign(per_body, per_body + nb);
  const bool c =
      ok(cudaMemcpy(g.rb_pos, body_pos4, 16 * (size_t)nb, cudaMemcpyHostToDevice), "upload") &&
      ok(cudaMemcpy(g.rb_vel, body_vel4, 16 * (size_t)nb, cudaMemcpyHostToDevice), "upload") &&
      ok(cudaMemcpy(g.rb_ang, body_ang4, 16 * (size_t)nb, cudaMemcpyHostToDevice), "upload") &&
      ok(cudaMemcpy(g.rb_quat, ident.data(), 16 * (size_t)nb, cudaMemcpyHostToDevice), "upload") &&
      ok(cudaMemcpy(g.rb_inertia, inv_inertia9, 36 * (size_t)nb, cudaMemcpyHostToDevice),
         "upload") &&
      ok(cudaMemcpy(g.rb_mass, mass, 4 * (size_t)nb, cudaMemcpyHostToDevice), "upload") &&
      ok(cudaMemcpy(g.rel, rel4, 16 * (size_t)n, cudaMemcpyHostToDevice), "upload") &&
      ok(cudaMemcpy(g.rb_index, rb_index, 4 * (size_t)n, cudaMemcpyHostToDevice), "upload");
  for (cudaEvent_t& e : g.ev) cudaEventCreate(&e);
  if (!c) {
    release();
    return 1;
  }
  return 0;
}

// One updateUniformGridDEM step; stage_ms[kStages] gets each stage's GPU-timeline time and
// *host_ms the step's wall time.  Returns 0 on success.
int ref_gpu_step(float* stage_ms, float* host_ms) {
  if (!g.n) return 1;
  const auto t0 = std::chrono::steady_clock::now();
  cudaEventRecord(g.ev[0], 0);
  setParameters(&g.prm);
  // Integrate_Rigid_Body_System_GPU (Particles/updateFunctions.cpp:2899-2949)
  glm::mat4* model_gpu = nullptr;
  glm::quat* cum_gpu = nullptr;
  if (!ok(cudaMalloc((void**)&model_gpu, sizeof(glm::mat4) * g.nb), "model matrices") ||
      !ok(cudaMalloc((void**)&cum_gpu, sizeof(glm::quat) * g.nb), "cumulative quaternions"))
    return 1;
  cudaMemcpy(cum_gpu, g.cum_quat.data(), sizeof(glm::quat) * g.nb, cudaMemcpyHostToDevice);
  GPUintegratorWrapper(g.rb_pos, g.rb_vel, g.rb_ang, g.rb_quat, g.rb_inertia, g.rb_cur_inertia,
                       model_gpu, cum_gpu, g.dt, g.rb_mass, g.nb, g.prm, kThreads);
  if (!ok(cudaDeviceSynchronize(), "GPUintegratorWrapper")) return 1;
  cudaMemcpy(g.cum_quat.data(), cum_gpu, sizeof(glm::quat) * g.nb, cudaMemcpyDeviceToHost);
  cudaMemcpy(g.model.data(), model_gpu, sizeof(glm::mat4) * g.nb, cudaMemcpyDeviceToHost);
  cudaFree(cum_gpu);
  cudaFree(model_gpu);
  computeGlobalAttributesWrapper(g.rb_pos, g.rb_vel, g.rel, g.pos, g.vel, g.rb_quat, g.rb_ang,
                                 g.rb_index, g.n, kThreads);
  if (!ok(cudaDeviceSynchronize(), "computeGlobalAttributesWrapper")) return 1;
  resetQuaternionWrapper(g.rb_quat, g.nb, kThreads);
  if (!ok(cudaDeviceSynchronize(), "resetQuaternionWrapper")) return 1;
  cudaEventRecord(g.ev[1], 0);
  cudaMemset(g.p_force, 0, sizeof(float) * 4 * g.n);
  cudaMemset(g.p_torque, 0, sizeof(float) * 4 * g.n);
  cudaEventRecord(g.ev[2], 0);
  // Find_And_Handle_Rigid_Body_Collisions_Uniform_Grid_DEM (RigidBodies/UniformGridUpdate.cpp:817-880)
  calc_hash();
  if (!ok(cudaDeviceSynchronize(), "calcHash")) return 1;
  cudaEventRecord(g.ev[3], 0);
  if (!sort_pairs()) return 1;
  cudaEventRecord(g.ev[4], 0);
  reorder();
  if (!ok(cudaDeviceSynchronize(), "reorderDataAndFindCellStart")) return 1;
  cudaEventRecord(g.ev[5], 0);
  const float3 lo = make_float3(0.f, 0.f, 0.f), hi = make_float3(1.f, 1.f, 1.f);
  FindAndHandleRigidBodyCollisionsUniformGridWrapper(g.rb_index, g.p_force, g.p_torque, g.color,
                                                     g.spos, g.svel, g.rel, lo, hi, g.index,
                                                     g.cell_start, g.cell_end, (uint)g.n, g.prm,
                                                     kThreads);
  if (!ok(cudaDeviceSynchronize(), "FindAndHandleRigidBodyCollisionsUniformGridWrapper"))
    return 1;
  cudaEventRecord(g.ev[6], 0);
  ReducePerParticleImpulses(g.rb_index, g.p_force, g.p_torque, g.rb_vel, g.rb_ang, g.rb_mass,
                            g.rb_inertia, g.per_body.data(), g.nb, g.n, kThreads);
  cudaEventRecord(g.ev[7], 0);
  if (!ok(cudaEventSynchronize(g.ev[7]), "step")) return 1;
  for (int i = 0; i < kStages; ++i) cudaEventElapsedTime(stage_ms + i, g.ev[i], g.ev[i + 1]);
  *host_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return ok(cudaGetLastError(), "step") ? 0 : 1;
}

// Body centres and velocities after the steps run so far (float4 each).
int ref_gpu_download(float* body_pos4, float* body_vel4) {
  if (!g.n) return 1;
  return ok(cudaMemcpy(body_pos4, g.rb_pos, 16 * (size_t)g.nb, cudaMemcpyDeviceToHost),
            "download") &&
                 ok(cudaMemcpy(body_vel4, g.rb_vel, 16 * (size_t)g.nb, cudaMemcpyDeviceToHost),
                    "download")
             ? 0
             : 1;
}

void ref_gpu_destroy() { release(); }

}  // extern "C"
