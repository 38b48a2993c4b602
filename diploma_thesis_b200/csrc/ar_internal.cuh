// Internal helpers shared by every translation unit of libarsim.so.
//
// Arithmetic convention: the library is compiled with -fmad=false, so every a*b+c below is
// a rounded multiply followed by a rounded add unless fmaf() is written explicitly.  The
// oracle (oracle/oracle.c, compiled with -ffp-contract=off) evaluates the same expressions
// in the same order, which is what makes the GPU results bit-identical to the oracle's
// float32 restatement wherever only + - * / sqrt are involved.
#pragma once
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

#include "../../include/arsim.h"

namespace ar {

constexpr uint32_t kEmpty = 0xffffffffu;  // empty grid cell (Kernels/particleKernels.cu:323)
constexpr int kNumSMs = 148;

// Device error word bits (ORed by kernels, read and cleared by ar_ctx_status).
enum : int {
  kErrTimeout = 1,   // a bounded spin wait gave up
  kErrNaN = 2,       // non-finite state detected
  kErrOverflow = 4,  // an output buffer was too small
};

// ---- float3/float4 helpers (own definitions; evaluation order is part of the contract) ----
__host__ __device__ __forceinline__ float3 mk3(float x, float y, float z) { return make_float3(x, y, z); }
__host__ __device__ __forceinline__ float3 xyz(float4 a) { return make_float3(a.x, a.y, a.z); }
__host__ __device__ __forceinline__ float3 add(float3 a, float3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
__host__ __device__ __forceinline__ float3 sub(float3 a, float3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
__host__ __device__ __forceinline__ float3 scl(float s, float3 a) { return mk3(s * a.x, s * a.y, s * a.z); }
__host__ __device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__host__ __device__ __forceinline__ float3 cross(float3 a, float3 b) {
  return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ float3 divs(float3 a, float s) { return mk3(a.x / s, a.y / s, a.z / s); }

// Rotate v by the unit quaternion q = (x, y, z, w):  t = 2 (q.xyz x v);  v' = v + w t + q.xyz x t.
__host__ __device__ __forceinline__ float3 quat_rotate(float4 q, float3 v) {
  float3 u = mk3(q.x, q.y, q.z);
  float3 t = scl(2.0f, cross(u, v));
  return add(add(v, scl(q.w, t)), cross(u, t));
}

// Row-major 3x3 times vector (m[0..2] = first row).
__host__ __device__ __forceinline__ float3 mat3_mul(const float* m, float3 v) {
  return mk3(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
             m[6] * v.x + m[7] * v.y + m[8] * v.z);
}

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

__device__ __forceinline__ void raise_error(int* err, int bits) {
  if (err) atomicOr(err, bits);
}

// Programmatic dependent launch: a kernel started with arh::launch_pdl may begin while the
// kernel before it on the stream is still finishing, so it calls pdl_wait() before it reads
// or writes anything that kernel (or earlier work) touches; the wait returns once the
// previous kernel has completed and its writes are visible.  In a kernel launched the
// ordinary way it returns at once.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

}  // namespace ar

// ---- host-side helpers ---------------------------------------------------------------------
namespace arh {
void set_error(const char* fmt, ...);
ar_status check_launch(const char* what);
inline cudaStream_t stream(ar_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }
inline unsigned grid_for(long n, int block) {
  long g = (n + block - 1) / block;
  return (unsigned)(g < 1 ? 1 : g);
}
#ifdef __CUDACC__
// Launch with programmatic stream serialisation: the kernel's blocks may be scheduled as the
// previous kernel's blocks retire (its launch latency overlaps that kernel's tail); the
// kernel must call ar::pdl_wait() before touching shared state.
template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
                       cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr{};
  attr.id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr.val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = &attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, args...);
}
#endif
}  // namespace arh

// Context: one per device.  Owns the device error word and a grow-only scratch arena that
// the stage entry points carve their temporaries from (no allocation in steady state).
struct ar_ctx {
  int device = 0;
  int* d_err = nullptr;        // device error word
  int* h_err = nullptr;        // pinned mirror
  void* scratch = nullptr;     // grow-only arena
  size_t scratch_bytes = 0;
  int num_sms = 148;
};

namespace arh {
// Ensure the context's scratch arena holds at least `bytes`; returns its base or null.
void* scratch(ar_ctx* ctx, size_t bytes);
// Every device and pinned-host allocation of the library goes through these, so that a test
// can make them fail on the host (ar_test_fail_allocations) and check each AR_ERR_OOM path.
cudaError_t dev_malloc(void** p, size_t bytes);
cudaError_t dev_malloc_async(void** p, size_t bytes, cudaStream_t st);
cudaError_t host_malloc(void** p, size_t bytes);
}  // namespace arh
