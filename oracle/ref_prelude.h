// Host prelude that lets the reference's CUDA kernel bodies compile as plain C++.
//
// TEST INFRASTRUCTURE ONLY. This header belongs to the oracle: it is used to build
// oracle/_ref/libref_cpu.so, the reference's own per-particle / per-body kernel bodies
// run in host loops. Nothing in the product (diploma_thesis_b200/) includes it.
//
// The CUDA runtime headers already give host definitions of float3/float4/uint3/dim3
// and make_*; this file supplies the few device intrinsics and built-in variables the
// extracted kernel bodies use, with the device semantics they have on the GPU:
//   threadIdx / blockIdx / blockDim / gridDim  -> thread_local variables the driver sets
//   __clz, __int2double_rn, __double2int_ru     -> exact integer / double equivalents
//   __fsqrt_rz                                  -> square root rounded toward zero
//   atomicAdd(int*)                             -> a sequentially consistent fetch-add
//   unary minus on a float3 rvalue              -> a const overload
//   min/max on float and unsigned               -> fminf/fmaxf and unsigned compare
//     (device code resolves min/max(float) to fminf/fmaxf; the reference's host
//      helper header only declares int versions, which would truncate floats)
#pragma once
#include <cuda_runtime.h>
#include <cmath>
#include <cstdint>

extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;

inline int __clz(int x) { return x == 0 ? 32 : __builtin_clz((unsigned)x); }
inline double __int2double_rn(int i) { return (double)i; }
inline int __double2int_ru(double d) { return (int)std::ceil(d); }
inline float __fsqrt_rz(float x) {
  float s = std::sqrt(x);
  if ((double)s * (double)s > (double)x) s = std::nextafter(s, 0.0f);
  return s;
}
inline int atomicAdd(int* p, int v) { return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST); }
inline void __threadfence() { __atomic_thread_fence(__ATOMIC_SEQ_CST); }
inline float min(float a, float b) { return std::fmin(a, b); }
inline float max(float a, float b) { return std::fmax(a, b); }
inline unsigned int min(unsigned int a, unsigned int b) { return a < b ? a : b; }
inline unsigned int max(unsigned int a, unsigned int b) { return a > b ? a : b; }
// helper_math.h's unary minus takes float3& (MSVC bound an rvalue to it at
// RigidBodies/UniformGridDEM.cu:284); a const overload gives the same negation for rvalues.
inline float3 operator-(const float3& a) { return make_float3(-a.x, -a.y, -a.z); }
