// (a6) scene AABB and (a7) 30/63-bit Morton codes.
#include "ar_internal.cuh"

namespace {

// The reference's `inf` is the int 0x7f800000 converted to float (BVHSource/createMortonCodes.cu:10,74,91).
constexpr float kInfInt = 2139095040.0f;

// Single-pass min/max over all four lanes: grid-stride float4 loads, warp shuffles, one
// block partial each, and the last block to finish folds the partials (fence + counter).
// min/max are order independent, so the result equals CUB's reduction for finite inputs.
__global__ void __launch_bounds__(256) aabb_kernel(const float4* __restrict__ pos, int n,
                                                   float4* __restrict__ partials,
                                                   unsigned* __restrict__ counter,
                                                   float4* __restrict__ out_min,
                                                   float4* __restrict__ out_max) {
  float lo[4] = {kInfInt, kInfInt, kInfInt, kInfInt};
  float hi[4] = {-kInfInt, -kInfInt, -kInfInt, -kInfInt};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 p = __ldg(pos + i);
    float v[4] = {p.x, p.y, p.z, p.w};
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      lo[c] = (v[c] < lo[c]) ? v[c] : lo[c];
      hi[c] = (v[c] > hi[c]) ? v[c] : hi[c];
    }
  }
#pragma unroll
  for (int c = 0; c < 4; ++c)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      float a = __shfl_xor_sync(0xffffffffu, lo[c], o);
      float b = __shfl_xor_sync(0xffffffffu, hi[c], o);
      lo[c] = (a < lo[c]) ? a : lo[c];
      hi[c] = (b > hi[c]) ? b : hi[c];
    }
  __shared__ float s_lo[8][4], s_hi[8][4];
  __shared__ bool s_last;
  const int w = threadIdx.x >> 5;
  if (ar::lane_id() == 0)
    for (int c = 0; c < 4; ++c) { s_lo[w][c] = lo[c]; s_hi[w][c] = hi[c]; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k)
      for (int c = 0; c < 4; ++c) {
        lo[c] = (s_lo[k][c] < lo[c]) ? s_lo[k][c] : lo[c];
        hi[c] = (s_hi[k][c] > hi[c]) ? s_hi[k][c] : hi[c];
      }
    partials[2 * blockIdx.x] = make_float4(lo[0], lo[1], lo[2], lo[3]);
    partials[2 * blockIdx.x + 1] = make_float4(hi[0], hi[1], hi[2], hi[3]);
    __threadfence();
    unsigned done = atomicAdd(counter, 1u);
    s_last = (done == gridDim.x - 1);
  }
  __syncthreads();
  if (s_last && threadIdx.x == 0) {
    __threadfence();
    float L[4] = {kInfInt, kInfInt, kInfInt, kInfInt};
    float H[4] = {-kInfInt, -kInfInt, -kInfInt, -kInfInt};
    for (unsigned b = 0; b < gridDim.x; ++b) {
      float4 a = __ldcg(partials + 2 * b), c4 = __ldcg(partials + 2 * b + 1);
      float av[4] = {a.x, a.y, a.z, a.w}, cv[4] = {c4.x, c4.y, c4.z, c4.w};
      for (int c = 0; c < 4; ++c) {
        L[c] = (av[c] < L[c]) ? av[c] : L[c];
        H[c] = (cv[c] > H[c]) ? cv[c] : H[c];
      }
    }
    *out_min = make_float4(L[0], L[1], L[2], L[3]);
    *out_max = make_float4(H[0], H[1], H[2], H[3]);
    *counter = 0;  // ready for the next call
  }
}

// Spread the low 10 bits of v so bit k moves to bit 3k (same result as the reference's
// multiply-and-mask expandBits, BVHSource/BVHkernels.cu:648-655).
__device__ __forceinline__ uint32_t spread10(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

// Spread the low 21 bits of v so bit k moves to bit 3k.
__device__ __forceinline__ uint64_t spread21(uint64_t v) {
  v &= 0x1fffffull;
  v = (v | (v << 32)) & 0x001f00000000ffffull;
  v = (v | (v << 16)) & 0x001f0000ff0000ffull;
  v = (v | (v << 8)) & 0x100f00f00f00f00full;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
  v = (v | (v << 2)) & 0x1249249249249249ull;
  return v;
}

// Normalised coordinate -> integer cell in [0, scale-1]: clamp(x*scale, 0, scale-1) then
// truncate (morton3D, BVHkernels.cu:659-668; device min/max are fminf/fmaxf).
__device__ __forceinline__ uint32_t quantise(float x, float scale, float top) {
  return (uint32_t)fminf(fmaxf(x * scale, 0.0f), top);
}

template <bool kDeviceBox>
__global__ void __launch_bounds__(256) morton30_kernel(const float4* __restrict__ pos, int n,
                                                       const float4* __restrict__ dmin,
                                                       const float4* __restrict__ dmax,
                                                       float4 hmin, float4 hmax,
                                                       uint32_t* __restrict__ codes,
                                                       int32_t* __restrict__ idx) {
  float4 mn = kDeviceBox ? *dmin : hmin;
  float4 mx = kDeviceBox ? *dmax : hmax;
  const float ex = mx.x - mn.x, ey = mx.y - mn.y, ez = mx.z - mn.z;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 p = __ldg(pos + i);
    float x = (p.x - mn.x) / ex;
    float y = (p.y - mn.y) / ey;
    float z = (p.z - mn.z) / ez;
    uint32_t xx = spread10(quantise(x, 1024.0f, 1023.0f));
    uint32_t yy = spread10(quantise(y, 1024.0f, 1023.0f));
    uint32_t zz = spread10(quantise(z, 1024.0f, 1023.0f));
    codes[i] = (xx << 2) | (yy << 1) | zz;
    if (idx) idx[i] = i;
  }
}

__global__ void __launch_bounds__(256) morton63_kernel(const float4* __restrict__ pos, int n,
                                                       const float4* __restrict__ dmin,
                                                       const float4* __restrict__ dmax,
                                                       uint64_t* __restrict__ codes,
                                                       int32_t* __restrict__ idx) {
  float4 mn = *dmin, mx = *dmax;
  const float ex = mx.x - mn.x, ey = mx.y - mn.y, ez = mx.z - mn.z;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 p = __ldg(pos + i);
    float x = (p.x - mn.x) / ex;
    float y = (p.y - mn.y) / ey;
    float z = (p.z - mn.z) / ez;
    uint64_t xx = spread21(quantise(x, 2097152.0f, 2097151.0f));
    uint64_t yy = spread21(quantise(y, 2097152.0f, 2097151.0f));
    uint64_t zz = spread21(quantise(z, 2097152.0f, 2097151.0f));
    codes[i] = (xx << 2) | (yy << 1) | zz;
    if (idx) idx[i] = i;
  }
}

unsigned stream_grid(const ar_ctx* ctx, long n, int block) {
  long g = (n + block - 1) / block;
  long cap = (long)ctx->num_sms * 8;
  if (g > cap) g = cap;
  return (unsigned)(g < 1 ? 1 : g);
}

}  // namespace

extern "C" {

ar_status ar_scene_aabb(ar_ctx* ctx, const float* pos4, int n, float* d_min4, float* d_max4,
                        ar_stream_t stream) {
  if (!ctx || (n > 0 && !pos4) || !d_min4 || !d_max4 || n < 0) return AR_ERR_INVALID_ARG;
  unsigned grid = stream_grid(ctx, n, 256);
  if (grid > 1024) grid = 1024;
  // scratch: [counter (256 B aligned)] [partials 2*grid float4]
  char* s = (char*)arh::scratch(ctx, 256 + sizeof(float4) * 2 * grid);
  if (!s) return AR_ERR_OOM;
  cudaStream_t st = arh::stream(stream);
  cudaMemsetAsync(s, 0, sizeof(unsigned), st);
  aabb_kernel<<<grid, 256, 0, st>>>((const float4*)pos4, n, (float4*)(s + 256), (unsigned*)s,
                                    (float4*)d_min4, (float4*)d_max4);
  return arh::check_launch("ar_scene_aabb");
}

ar_status ar_morton30(ar_ctx* ctx, const float* pos4, int n, const float* d_min4,
                      const float* d_max4, uint32_t* codes, int32_t* idx, ar_stream_t stream) {
  if (!ctx || n < 0 || (n > 0 && (!pos4 || !codes || !d_min4 || !d_max4)))
    return AR_ERR_INVALID_ARG;
  if (n == 0) return AR_OK;
  float4 z = make_float4(0, 0, 0, 0);
  morton30_kernel<true><<<stream_grid(ctx, n, 256), 256, 0, arh::stream(stream)>>>(
      (const float4*)pos4, n, (const float4*)d_min4, (const float4*)d_max4, z, z, codes, idx);
  return arh::check_launch("ar_morton30");
}

ar_status ar_morton30_box(ar_ctx* ctx, const float* pos4, int n, const float h_min4[4],
                          const float h_max4[4], uint32_t* codes, int32_t* idx,
                          ar_stream_t stream) {
  if (!ctx || n < 0 || !h_min4 || !h_max4 || (n > 0 && (!pos4 || !codes)))
    return AR_ERR_INVALID_ARG;
  if (n == 0) return AR_OK;
  float4 mn = make_float4(h_min4[0], h_min4[1], h_min4[2], h_min4[3]);
  float4 mx = make_float4(h_max4[0], h_max4[1], h_max4[2], h_max4[3]);
  morton30_kernel<false><<<stream_grid(ctx, n, 256), 256, 0, arh::stream(stream)>>>(
      (const float4*)pos4, n, nullptr, nullptr, mn, mx, codes, idx);
  return arh::check_launch("ar_morton30_box");
}

ar_status ar_morton63(ar_ctx* ctx, const float* pos4, int n, const float* d_min4,
                      const float* d_max4, uint64_t* codes, int32_t* idx, ar_stream_t stream) {
  if (!ctx || n < 0 || (n > 0 && (!pos4 || !codes || !d_min4 || !d_max4)))
    return AR_ERR_INVALID_ARG;
  if (n == 0) return AR_OK;
  morton63_kernel<<<stream_grid(ctx, n, 256), 256, 0, arh::stream(stream)>>>(
      (const float4*)pos4, n, (const float4*)d_min4, (const float4*)d_max4, codes, idx);
  return arh::check_launch("ar_morton63");
}

}  // extern "C"
