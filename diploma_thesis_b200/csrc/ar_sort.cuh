// Internal interface of the onesweep radix sort, used by the fused step pipeline.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/arsim.h"

struct ar_ctx;

namespace ar_sort {

constexpr int kMaxPasses = 8;
constexpr int kMaxRadix = 512;  // digits are 8 bits wide, or 9 where that saves a pass

// Digit passes of a sort over key bits [begin, end): as few passes as 9-bit digits allow,
// 8-bit digits where the bits suffice and 9-bit digits for the last (bits - 8 * passes)
// passes otherwise (24 bits: 8, 8, 8; 25 bits: 8, 8, 9; 30 bits: 8, 8, 8, 6; 63 bits: 9 x 7).
struct Plan {
  int passes;
  int shift[kMaxPasses];
  int bits[kMaxPasses];
};
inline Plan make_plan(int begin_bit, int end_bit) {
  Plan p{};
  const int total = end_bit - begin_bit;
  p.passes = total <= 0 ? 0 : (total + 8) / 9;
  const int wide = total - 8 * p.passes;  // > 0: passes that take 9 bits
  int shift = begin_bit;
  for (int i = 0; i < p.passes; ++i) {
    int b = 8;
    if (wide > 0 && i >= p.passes - wide) b = 9;
    if (wide <= 0 && i == p.passes - 1) b = total - 8 * (p.passes - 1);
    p.shift[i] = shift;
    p.bits[i] = b;
    shift += b;
  }
  return p;
}

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
// (identity).  Device errors go to ctx->d_err.  match_rank: rank 8-bit digits with warp
// match.any (faster when a warp's keys share few digits, as cell keys in particle order do).
ar_status sort_u32(ar_ctx* ctx, const uint32_t* keys_in, const uint32_t* vals_in,
                   uint32_t* keys_out, uint32_t* vals_out, int n, int begin_bit, int end_bit,
                   cudaStream_t st, void* ws, size_t ws_bytes, bool external_hist = false,
                   bool match_rank = false);

// The same for u64 keys (histogram computed inside; workspace layout(n, 8, passes)).
ar_status sort_u64(ar_ctx* ctx, const uint64_t* keys_in, const uint32_t* vals_in,
                   uint64_t* keys_out, uint32_t* vals_out, int n, int begin_bit, int end_bit,
                   cudaStream_t st, void* ws, size_t ws_bytes);

// Bytes at the head of the workspace that must be zero before a sort whose histogram is
// accumulated externally (histograms, tile counters, look-back status).
size_t clear_bytes(long n, int passes);

// Histogram of `key` for every pass of `plan` into a shared [kMaxPasses][kMaxRadix] block
// histogram (then hist_flush), with one shared-memory atomic per distinct digit per warp (the
// lanes holding the same digit are counted by their lowest lane): particles of a body are
// adjacent in the original order and mostly share digits, so this removes most same-address
// contention.
__device__ __forceinline__ void hist_count_warp(uint32_t (*s_hist)[kMaxRadix], uint32_t key,
                                                const Plan& plan) {
  const uint32_t active = __activemask();
  const int lane = threadIdx.x & 31;
  for (int p = 0; p < plan.passes; ++p) {
    const uint32_t d = (key >> plan.shift[p]) & ((1u << plan.bits[p]) - 1);
    const uint32_t peers = __match_any_sync(active, d);
    if (lane == __ffs(peers) - 1) atomicAdd(&s_hist[p][d], (uint32_t)__popc(peers));
  }
}
// Block histogram -> workspace head (ws + 0 holds uint32 [kMaxPasses][kMaxRadix]).
__device__ __forceinline__ void hist_flush(uint32_t (*s_hist)[kMaxRadix], uint32_t* ws_hist,
                                           int passes) {
  for (int i = threadIdx.x; i < passes * kMaxRadix; i += blockDim.x) {
    uint32_t v = (&s_hist[0][0])[i];
    if (v) atomicAdd(ws_hist + i, v);
  }
}

// Kernel launches one sort call issues (memset and histogram count when not external).
int launches(int begin_bit, int end_bit, bool external_hist = false);

}  // namespace ar_sort
