// Internal interface of the onesweep radix sort, used by the fused step pipeline.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/arsim.h"

struct ar_ctx;

namespace ar_sort {

constexpr int kMaxPasses = 8;

// Per-device kernel attributes (dynamic shared memory opt-in); called by ar_ctx_create so
// that no attribute call ever happens inside a graph capture.
void init();

// Byte offsets of the sort's workspace pieces (256-byte aligned).
struct Layout {
  size_t hist, counters, status, tmp_keys, tmp_vals, total;
};
Layout layout(long n, size_t key_bytes, int passes);

void iota(uint32_t* v, int n, cudaStream_t st);

// Sort u32 (key, value) pairs by bits [begin_bit, end_bit) into keys_out/vals_out using the
// caller's workspace (at least layout(n, 4, passes).total bytes).  vals_in may be null
// (identity).  Device errors go to ctx->d_err.
ar_status sort_u32(ar_ctx* ctx, const uint32_t* keys_in, const uint32_t* vals_in,
                   uint32_t* keys_out, uint32_t* vals_out, int n, int begin_bit, int end_bit,
                   cudaStream_t st, void* ws, size_t ws_bytes, bool external_hist = false);

// The same for u64 keys (histogram computed inside; workspace layout(n, 8, passes)).
ar_status sort_u64(ar_ctx* ctx, const uint64_t* keys_in, const uint32_t* vals_in,
                   uint64_t* keys_out, uint32_t* vals_out, int n, int begin_bit, int end_bit,
                   cudaStream_t st, void* ws, size_t ws_bytes);

// Bytes at the head of the workspace that must be zero before a sort whose histogram is
// accumulated externally (histograms, tile counters, look-back status).
size_t clear_bytes(long n, int passes);

// Histogram of `key` for every pass into the workspace head (call from a kernel that holds
// a shared [kMaxPasses][256] block histogram; see hist_flush).  Digit width 8, last pass
// `last_bits` wide.
__device__ __forceinline__ void hist_count(uint32_t (*s_hist)[256], uint32_t key, int begin_bit,
                                           int passes, int last_bits) {
  for (int p = 0; p < passes; ++p) {
    uint32_t mask = (p == passes - 1) ? ((1u << last_bits) - 1) : 0xffu;
    atomicAdd(&s_hist[p][(key >> (begin_bit + 8 * p)) & mask], 1u);
  }
}
// hist_count with one shared-memory atomic per distinct digit per warp (the lanes holding the
// same digit are counted by their lowest lane): particles of a body are adjacent in the
// original order and mostly share digits, so this removes most same-address contention.
__device__ __forceinline__ void hist_count_warp(uint32_t (*s_hist)[256], uint32_t key,
                                                int begin_bit, int passes, int last_bits) {
  const uint32_t active = __activemask();
  const int lane = threadIdx.x & 31;
  for (int p = 0; p < passes; ++p) {
    const uint32_t mask = (p == passes - 1) ? ((1u << last_bits) - 1) : 0xffu;
    const uint32_t d = (key >> (begin_bit + 8 * p)) & mask;
    const uint32_t peers = __match_any_sync(active, d);
    if (lane == __ffs(peers) - 1) atomicAdd(&s_hist[p][d], (uint32_t)__popc(peers));
  }
}
// Block histogram -> workspace head (ws + 0 holds uint32 [kMaxPasses][256]).
__device__ __forceinline__ void hist_flush(uint32_t (*s_hist)[256], uint32_t* ws_hist,
                                           int passes) {
  for (int i = threadIdx.x; i < passes * 256; i += blockDim.x) {
    uint32_t v = (&s_hist[0][0])[i];
    if (v) atomicAdd(ws_hist + i, v);
  }
}

// Kernel launches one sort call issues (memset and histogram count when not external).
int launches(int begin_bit, int end_bit, bool external_hist = false);

}  // namespace ar_sort
