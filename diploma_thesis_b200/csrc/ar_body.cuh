// Per-body device helpers shared by the stage kernels and the fused step.
#pragma once
#include "ar_internal.cuh"

namespace ar_body {

// Fixed-order sum of pf/pt over [s, e) by the calling warp: lane l adds elements s+l,
// s+l+32, ... in order, then the lanes combine with a xor-shuffle tree (16, 8, 4, 2, 1),
// each lane adding its partner's value to its own.  Every lane returns lane 0's result.
__device__ __forceinline__ void warp_segment_sum(const float4* __restrict__ pf,
                                                 const float4* __restrict__ pt, int s, int e,
                                                 float3* f_out, float3* t_out) {
  const int lane = ar::lane_id();
  float fx = 0.f, fy = 0.f, fz = 0.f, tx = 0.f, ty = 0.f, tz = 0.f;
  for (int i = s + lane; i < e; i += 32) {
    const float4 a = __ldcs(pf + i);
    const float4 b = __ldcs(pt + i);
    fx += a.x; fy += a.y; fz += a.z;
    tx += b.x; ty += b.y; tz += b.z;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    fx += __shfl_xor_sync(0xffffffffu, fx, o);
    fy += __shfl_xor_sync(0xffffffffu, fy, o);
    fz += __shfl_xor_sync(0xffffffffu, fz, o);
    tx += __shfl_xor_sync(0xffffffffu, tx, o);
    ty += __shfl_xor_sync(0xffffffffu, ty, o);
    tz += __shfl_xor_sync(0xffffffffu, tz, o);
  }
  *f_out = ar::mk3(__shfl_sync(0xffffffffu, fx, 0), __shfl_sync(0xffffffffu, fy, 0),
                   __shfl_sync(0xffffffffu, fz, 0));
  *t_out = ar::mk3(__shfl_sync(0xffffffffu, tx, 0), __shfl_sync(0xffffffffu, ty, 0),
                   __shfl_sync(0xffffffffu, tz, 0));
}

}  // namespace ar_body
