// Re-sort of the cell keys from the previous step's order.
//
// The grid step needs the particles ordered by (cell key, particle index): the stable sort of
// the keys in particle order that sortParticles (Kernels/particleKernelWrappers.cu:419-534)
// produces.  Between two steps only a small share of the particles changes cell (about 1 % per
// step on the 2M-particle pile), so the previous step's order, which is sorted by
// (old key, index), is almost the new one.  The four kernels below turn it into the new order
// exactly, whatever the number of particles that moved:
//
//   leavers_kernel  over the previous order, one tile of kTile positions per block: a
//                   particle whose key changed is a mover; a bit per position marks it, and
//                   the tile stores its mover count and its movers (new key, index), counted
//                   per key bucket (key >> bshift).
//   bucket_kernel   one warp per tile of kTile old positions: the tile's movers into their
//                   buckets' ranges, and the tile's header for place_kernel; every block scans
//                   the bucket counts and the tile counts it needs itself.
//   bucket_sort_kernel  each bucket sorted by (key, index): one warp per bucket, ranks by
//                   comparison (in registers up to 32 movers, in shared memory up to 256, in
//                   global memory beyond; buckets usually hold a few movers).
//   place_kernel    over the previous order.  A stayer (a particle that kept its key) at old
//                   position j has r = j - (movers before j) stayers before it in the new
//                   order too (their keys did not change and the old order is sorted), and A =
//                   (movers with a smaller (key, index)) movers before it, so it goes to r + A.
//                   Mover i (in sorted order) lies between the stayers whose A is <= i and
//                   those whose A is > i: the stayer s with A(previous stayer) <= i < A(s)
//                   writes it to r(s) + i, and the movers above every stayer go to (n - m) + i.
//
// (Finding the movers in the key kernel instead, from each particle's previous key, needs
// each particle's previous position: keeping that inverse permutation costs the scatter
// kernel more scattered stores than this pass costs.)
//
// Every position written is below n by construction (r + A <= (n - m - 1) + m), so a previous
// order that were not a sorted permutation would give a wrong order, never a stray write; the
// scatter kernel copies each step's order into the previous-order buffers, so it always is one.
#pragma once

#include <cstdint>

#include "ar_internal.cuh"

namespace ar_resort {

constexpr int kThreads = 256;
constexpr int kRows = 8;                  // positions per thread and tile
constexpr int kTile = kThreads * kRows;   // positions of the previous order per tile
constexpr int kWarps = kThreads / 32;
constexpr int kBucketLog2 = 12;           // at most 2^12 mover buckets
constexpr int kHeadWords = 4;             // counters at the head of the cleared region
constexpr int kWindow = 256;              // sorted movers a placement tile stages in shared memory
// tile header flags
constexpr uint32_t kHasPrev = 1;   // a stayer lies before the tile (its last one: thead[2t + 1])
constexpr uint32_t kTailOwner = 2; // the tile writes the movers above every stayer
constexpr uint32_t kNoStayers = 4; // no stayer at all: those movers start at 0

// Device workspace.  One region holds ctr[kHeadWords] (ctr[3] = m, written by bucket_kernel),
// bcount, bfill (kMaxBuckets each) -- zeroed by the step's first kernel (cleared_words) -- then
// tcount and bits (written whole by leavers_kernel).
constexpr int kMaxBuckets = 1 << kBucketLog2;
struct Work {
  uint32_t* head;
  uint32_t* bits;     // mover bit per position of the previous order (ceil(n / 32) words)
  uint32_t* tcount;   // movers per tile
  uint4* thead;       // per tile: {w0, w1, movers before the tile, flags}, {previous stayer}
  uint32_t* bstart;   // exclusive prefix of the bucket counts, [nb] = m
  uint2* local;       // movers of tile t at [t * kTile, t * kTile + tcount[t]), any order
  uint2* grouped;     // movers grouped by bucket
  uint2* movers;      // movers sorted by (key, index) (may share memory with local)
  int nb;             // buckets (a power of two)
  int bshift;         // bucket of key k: k >> bshift
  __host__ __device__ uint32_t* ctr() const { return head; }
  __host__ __device__ uint32_t* bcount() const { return head + kHeadWords; }
  __host__ __device__ uint32_t* bfill() const { return head + kHeadWords + kMaxBuckets; }
};

inline long tiles_for(long n) { return (n + kTile - 1) / kTile; }
inline long round4(long x) { return (x + 3) & ~3l; }
// Layout of the region for a capacity of cap particles; the words the step's first kernel
// clears.
inline size_t tcount_offset() { return (size_t)kHeadWords + 2 * (size_t)kMaxBuckets; }
inline size_t bits_offset(long cap) { return tcount_offset() + round4(tiles_for(cap) + 1); }
inline size_t region_words(long cap) { return bits_offset(cap) + round4(cap / 32 + 1); }
inline size_t cleared_words() { return tcount_offset(); }

__device__ __forceinline__ unsigned long long composite(uint32_t key, uint32_t idx) {
  return ((unsigned long long)key << 32) | idx;
}
__device__ __forceinline__ unsigned long long composite(uint2 e) { return composite(e.x, e.y); }

// 16-byte asynchronous copy global -> shared (cp.async); src_bytes < 16 zero-fills the rest and
// reads only src_bytes (the source address is then clamped by the caller).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// Stage a tile's old keys, indices (and mover bits) in shared memory: 16-byte copies, positions
// from n on read as 0.
__device__ __forceinline__ void stage_tile(const uint32_t* __restrict__ pk,
                                           const uint32_t* __restrict__ pv,
                                           const uint32_t* __restrict__ bits, long base, int n,
                                           uint32_t* s_k, uint32_t* s_v, uint32_t* s_bits) {
  for (int c = threadIdx.x; c < kTile / 4; c += kThreads) {
    const long j = base + 4 * c;
    const int nbytes = (int)max(0l, min(16l, 4 * ((long)n - j)));
    cp_async16(s_k + 4 * c, nbytes ? pk + j : pk, nbytes);
    cp_async16(s_v + 4 * c, nbytes ? pv + j : pv, nbytes);
  }
  if (s_bits && threadIdx.x < kTile / 128) {  // kTile / 32 words, 4 per copy
    const long w0 = base / 32 + 4 * threadIdx.x, nw = ((long)n + 31) / 32;
    const int nbytes = (int)max(0l, min(16l, 4 * (nw - w0)));
    cp_async16(s_bits + 4 * threadIdx.x, nbytes ? bits + w0 : bits, nbytes);
  }
  cp_async_wait_all();
}

// Exclusive scan of a[0, count) into out[0, count], out[count] = total, by one block of
// kThreads threads, in chunks of kThreads * kScanPer values; each thread loads its kScanPer
// consecutive values of a chunk together (one round trip), reading through L2 (the counts were
// written by other blocks).
constexpr int kScanPer = 16;
__device__ void block_scan(const uint32_t* a, uint32_t* out, int count) {
  __shared__ uint32_t s_warp[kWarps];
  __shared__ uint32_t s_carry;
  const int lane = ar::lane_id(), warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_carry = 0;
  for (int c0 = 0; c0 < count; c0 += kThreads * kScanPer) {
    const int lo = c0 + threadIdx.x * kScanPer;
    uint32_t v[kScanPer], t = 0;
#pragma unroll
    for (int q = 0; q < kScanPer; ++q) v[q] = lo + q < count ? __ldcg(a + lo + q) : 0u;
#pragma unroll
    for (int q = 0; q < kScanPer; ++q) t += v[q];
    uint32_t incl = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    uint32_t before = s_carry, total = 0;
#pragma unroll
    for (int q = 0; q < kWarps; ++q) {
      const uint32_t x = s_warp[q];
      before += q < warp ? x : 0u;
      total += x;
    }
    uint32_t run = before + incl - t;
#pragma unroll
    for (int q = 0; q < kScanPer; ++q) {
      if (lo + q < count) out[lo + q] = run;
      run += v[q];
    }
    __syncthreads();
    if (threadIdx.x == 0) s_carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) out[count] = s_carry;
}

// ---- movers of the previous order -----------------------------------------------------------
// The tile's old keys and indices are staged in shared memory (asynchronous 16-byte copies), so
// that few values stay in registers and every tile of the pile runs in one wave.
__global__ void __launch_bounds__(kThreads, 7) leavers_kernel(
    const uint32_t* __restrict__ pk, const uint32_t* __restrict__ pv,
    const uint32_t* __restrict__ keys, int n, Work w) {
  ar::pdl_wait();
  __shared__ __align__(16) uint32_t s_k[kTile];
  __shared__ __align__(16) uint32_t s_v[kTile];
  __shared__ uint32_t s_warp[kWarps];
  const int lane = ar::lane_id(), warp = threadIdx.x >> 5;
  const long base = (long)blockIdx.x * kTile;
  stage_tile(pk, pv, nullptr, base, n, s_k, s_v, nullptr);
  __syncthreads();
  uint32_t kn[kRows];
#pragma unroll
  for (int u = 0; u < kRows; ++u) {
    const int off = u * kThreads + threadIdx.x;
    if (base + off < n) kn[u] = __ldg(keys + s_v[off]);
  }
  uint32_t ball[kRows], count = 0;
#pragma unroll
  for (int u = 0; u < kRows; ++u) {
    const int off = u * kThreads + threadIdx.x;
    ball[u] = __ballot_sync(0xffffffffu, base + off < n && kn[u] != s_k[off]);
    const long word0 = base + u * kThreads + warp * 32;  // first position of the warp's word
    if (lane == 0 && word0 < n) w.bits[word0 >> 5] = ball[u];
    count += __popc(ball[u]);
  }
  if (lane == 0) s_warp[warp] = count;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
    for (int q = 0; q < kWarps; ++q) {
      const uint32_t c = s_warp[q];
      s_warp[q] = t;
      t += c;
    }
    w.tcount[blockIdx.x] = t;
  }
  __syncthreads();
  uint32_t off = (uint32_t)base + s_warp[warp];
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
  for (int u = 0; u < kRows; ++u) {
    if (ball[u] >> lane & 1u) {
      w.local[off + __popc(ball[u] & lt)] = make_uint2(kn[u], s_v[u * kThreads + threadIdx.x]);
      atomicAdd(w.bcount() + (kn[u] >> w.bshift), 1u);
    }
    off += __popc(ball[u]);
  }
}

// ---- movers into their buckets, tile headers -----------------------------------------------
// One warp per tile.  Every block scans the bucket counts into shared memory and sums the tile
// counts before its tiles (and all of them, m); block 0 also stores the bucket starts and m.
// The loads that do not need the scans (the tile's first 32 movers, its first and last old
// keys, the last stayer before it) are issued before them.
__global__ void __launch_bounds__(kThreads) bucket_kernel(const uint32_t* __restrict__ pk,
                                                          const uint32_t* __restrict__ pv,
                                                          int n, int tiles, Work w) {
  ar::pdl_wait();
  __shared__ uint32_t s_bstart[(1 << kBucketLog2) + 1];
  __shared__ uint32_t s_red[2][kWarps];
  __shared__ uint32_t s_tc[kWarps];  // movers of the block's tiles
  const int lane = ar::lane_id(), warp = threadIdx.x >> 5;
  const int t0 = blockIdx.x * kWarps;
  const int t = t0 + warp;
  const bool live = t < tiles;
  const long base = (long)t * kTile, end = min((long)n, base + kTile);
  const uint2* __restrict__ src = w.local + (size_t)t * kTile;
  // issued early: the tile's first 32 mover slots (only those below the tile's length, so
  // within the particle count), its first and last old keys, the last stayer before it
  uint2 e0 = make_uint2(0u, 0u);
  uint32_t kfirst = 0, klast = 0;
  uint2 prev = make_uint2(0u, 0u);
  bool has_prev = false;
  if (live) {
    if (lane < end - base) e0 = src[lane];
    if (lane == 0) {
      kfirst = __ldg(pk + base);
      klast = __ldg(pk + end - 1);
    } else if (lane == 1 && t > 0) {
      long q = t - 1;
      while (q > 0 && __ldcg(w.tcount + q) == (uint32_t)kTile) --q;  // tiles of movers only
      for (long wi = (q + 1) * (kTile / 32) - 1; wi >= q * (kTile / 32); --wi) {
        const uint32_t stay = ~__ldcg(w.bits + wi);  // earlier tiles are full
        if (stay) {
          const long j = wi * 32 + 31 - __clz(stay);
          prev = make_uint2(__ldg(pk + j), __ldg(pv + j));
          has_prev = true;
          break;
        }
      }
    }
  }
  uint32_t before = 0, total = 0;
  for (int i = threadIdx.x; i < tiles; i += kThreads) {
    const uint32_t c = __ldcg(w.tcount + i);
    total += c;
    before += i < t0 ? c : 0u;
    if (i >= t0 && i < t0 + kWarps) s_tc[i - t0] = c;
  }
  block_scan(w.bcount(), s_bstart, w.nb);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    before += __shfl_xor_sync(0xffffffffu, before, o);
    total += __shfl_xor_sync(0xffffffffu, total, o);
  }
  if (lane == 0) {
    s_red[0][warp] = before;
    s_red[1][warp] = total;
  }
  __syncthreads();
  uint32_t m = 0;
  before = 0;
#pragma unroll
  for (int q = 0; q < kWarps; ++q) {
    before += s_red[0][q];
    m += s_red[1][q];
  }
  if (blockIdx.x == 0) {
    for (int i = threadIdx.x; i <= w.nb; i += kThreads) w.bstart[i] = s_bstart[i];
    if (threadIdx.x == 0) w.ctr()[3] = m;
  }
  if (!live) return;
  const uint32_t cnt = s_tc[warp];
  uint32_t lead = before;  // movers before tile t
  for (int q = 0; q < warp; ++q) lead += s_tc[q];
  for (uint32_t i = lane; i < cnt; i += 32) {
    const uint2 e = i < 32 ? e0 : src[i];
    const uint32_t b = e.x >> w.bshift;
    const uint32_t slot = atomicAdd(w.bfill() + b, 1u);
    w.grouped[s_bstart[b] + slot] = e;
  }
  has_prev = __shfl_sync(0xffffffffu, has_prev, 1);
  prev.x = __shfl_sync(0xffffffffu, prev.x, 1);
  prev.y = __shfl_sync(0xffffffffu, prev.y, 1);
  if (lane == 0) {
    const uint32_t len = (uint32_t)(end - base);
    const uint32_t w0 = s_bstart[kfirst >> w.bshift];
    const uint32_t w1 = s_bstart[(klast >> w.bshift) + 1];
    uint32_t flags = 0;
    if ((uint32_t)base > lead && has_prev) flags |= kHasPrev;  // some stayer lies before
    const uint32_t stay_here = len - cnt;
    const uint32_t stay_after = (uint32_t)(n - end) - (m - (lead + cnt));
    if (stay_after == 0 && stay_here > 0) flags |= kTailOwner;
    if ((uint32_t)n == m && t == 0) flags |= kTailOwner | kNoStayers;
    w.thead[2 * t] = make_uint4(w0, max(w0, w1), lead, flags);
    w.thead[2 * t + 1] = make_uint4(prev.x, prev.y, 0u, 0u);
  }
}

// ---- each bucket sorted by (key, index) into w.movers --------------------------------------
// One warp per bucket; a mover's rank is the number of the bucket's movers with a smaller (key,
// index) (they are distinct).  Up to 32 movers: one per lane, compared through shuffles; up to
// kWarpStage: staged in the warp's shared memory and compared there; beyond: compared in
// global memory.  (Sorting chunks of 32 and merging them by binary searches was measured
// slower for the buckets of the 2M-particle pile, at most ~130 movers.)
constexpr int kWarpStage = 256;
__global__ void __launch_bounds__(kThreads) bucket_sort_kernel(Work w) {
  ar::pdl_wait();
  __shared__ unsigned long long s_stage[kWarps][kWarpStage];
  const int lane = ar::lane_id();
  unsigned long long* stage = s_stage[threadIdx.x >> 5];
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < w.nb; b += warps) {
    const uint32_t lo = __ldg(w.bstart + b), s = __ldg(w.bstart + b + 1) - lo;
    if (s == 0) continue;
    const uint2* __restrict__ g = w.grouped + lo;
    if (s <= 32) {
      const uint2 e = lane < (int)s ? g[lane] : make_uint2(0xffffffffu, 0xffffffffu);
      const unsigned long long ce = composite(e);
      uint32_t rank = 0;
      for (uint32_t t = 0; t < s; ++t) rank += __shfl_sync(0xffffffffu, ce, t) < ce;
      if (lane < (int)s) w.movers[lo + rank] = e;
    } else if (s <= (uint32_t)kWarpStage) {
      for (uint32_t i = lane; i < s; i += 32) stage[i] = composite(g[i]);
      __syncwarp();
      for (uint32_t i = lane; i < s; i += 32) {
        const unsigned long long ce = stage[i];
        uint32_t rank = 0;
        for (uint32_t t = 0; t < s; ++t) rank += stage[t] < ce;
        w.movers[lo + rank] = make_uint2((uint32_t)(ce >> 32), (uint32_t)ce);
      }
      __syncwarp();
    } else {
      for (uint32_t i = lane; i < s; i += 32) {
        const uint2 e = g[i];
        const unsigned long long ce = composite(e);
        uint32_t rank = 0;
        for (uint32_t t = 0; t < s; ++t) rank += composite(g[t]) < ce;
        w.movers[lo + rank] = e;
      }
    }
  }
}

// ---- every particle to its place in the new order -------------------------------------------
// Counting instead of searching: the movers that can lie below some stayer of the tile are
// those of the buckets from the tile's first old key to its last, [w0, w1) in sorted order
// (every mover below w0 has a smaller key than any particle of the tile, every one from w1 on
// a larger one); the tile stages them (up to kWindow) in shared memory.  Each is placed among
// the tile's old entries (sorted, also staged) by a binary search and counted at the first
// stayer above it; the inclusive prefix sum of the counts is then A - w0 for every stayer, and
// the exclusive one the A of the previous stayer of the tile, so the movers between two
// stayers are [A_excl, A).  For the tile's first stayer the previous stayer is the last one of
// an earlier tile (from the header) and the movers below A are walked down while they lie
// above it.  Per-position values live in shared memory, not registers, so that every tile of
// the pile runs in one wave.
__global__ void __launch_bounds__(kThreads, 7) place_kernel(
    const uint32_t* __restrict__ pk, const uint32_t* __restrict__ pv, int n, Work w,
    uint32_t* __restrict__ out_k, uint32_t* __restrict__ out_v, int* __restrict__ err) {
  ar::pdl_wait();
  __shared__ __align__(16) uint32_t s_k[kTile];     // old keys of the tile
  __shared__ __align__(16) uint32_t s_v[kTile];     // old indices of the tile
  __shared__ __align__(16) uint32_t s_bits[kTile / 32];  // mover bits of the tile
  __shared__ uint32_t s_cnt[kTile];  // movers counted at each stayer, then in-warp prefix
  __shared__ unsigned long long s_win[kWindow];
  __shared__ uint32_t s_lv[kRows * kWarps];  // movers per (row, warp), then exclusive prefix
  __shared__ uint32_t s_cs[kRows * kWarps];  // counts per (row, warp), then exclusive prefix
  __shared__ uint32_t s_end;
  const int lane = ar::lane_id(), warp = threadIdx.x >> 5;
  const int tile = blockIdx.x;
  const long base = (long)tile * kTile;
  const int len = (int)(min((long)n, base + kTile) - base);
  stage_tile(pk, pv, w.bits, base, n, s_k, s_v, s_bits);
  const uint4 h = w.thead[2 * tile];
  const uint32_t m = __ldcg(w.ctr() + 3);
  const uint32_t w0 = min(h.x, m), w1 = max(w0, min(h.y, m));
  const uint32_t wn = min((uint32_t)kWindow, w1 - w0);
  for (uint32_t i = threadIdx.x; i < wn; i += kThreads) s_win[i] = composite(w.movers[w0 + i]);
#pragma unroll
  for (int u = 0; u < kRows; ++u) s_cnt[u * kThreads + threadIdx.x] = 0u;
  __syncthreads();
  auto mover = [&](uint32_t i) {
    return i - w0 < wn ? s_win[i - w0] : composite(w.movers[i]);
  };
  for (uint32_t i = w0 + threadIdx.x; i < w1; i += kThreads) {
    const unsigned long long c = mover(i);
    int lo = 0, hi = len;  // first position whose old entry is above the mover
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (composite(s_k[mid], s_v[mid]) < c) lo = mid + 1; else hi = mid;
    }
    // on to the first stayer at or after lo: a clear bit of the tile's mover bits (a body
    // whose particles are consecutive in the old order moves as one run of up to 64)
    if (lo < len) {
      int wi = lo >> 5;
      uint32_t stay = ~s_bits[wi] & (0xffffffffu << (lo & 31));
      while (!stay && ++wi < kTile / 32) stay = ~s_bits[wi];
      lo = stay ? (wi << 5) + __ffs(stay) - 1 : len;
    }
    if (lo < len) atomicAdd(s_cnt + lo, 1u);
  }
  __syncthreads();
  // per (row, warp): mover count, and the in-warp inclusive sum of the counts in s_cnt's place
  // (the count itself is re-derived from the neighbour's sum)
#pragma unroll
  for (int u = 0; u < kRows; ++u) {
    const int off = u * kThreads + threadIdx.x;
    uint32_t x = s_cnt[off];
    if (__any_sync(0xffffffffu, x != 0u)) {  // most rows have no mover counted
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      s_cnt[off] = x;  // in-warp inclusive sum
    }
    if (lane == 31) {
      s_lv[u * kWarps + warp] = __popc(s_bits[off >> 5]);
      s_cs[u * kWarps + warp] = x;
    }
  }
  __syncthreads();
  if (threadIdx.x < 32) {  // exclusive prefix sums over the kRows * kWarps = 64 groups
    const uint32_t c0 = s_lv[2 * lane], c1 = s_lv[2 * lane + 1];
    const uint32_t d0 = s_cs[2 * lane], d1 = s_cs[2 * lane + 1];
    uint32_t ci = c0 + c1, di = d0 + d1;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, ci, o);
      const uint32_t z = __shfl_up_sync(0xffffffffu, di, o);
      if (lane >= o) {
        ci += y;
        di += z;
      }
    }
    const uint32_t cx = ci - c0 - c1, dx = di - d0 - d1;
    s_lv[2 * lane] = cx;
    s_lv[2 * lane + 1] = cx + c0;
    s_cs[2 * lane] = dx;
    s_cs[2 * lane + 1] = dx + d0;
    if (lane == 31) s_end = w0 + di;
  }
  __syncthreads();
  const uint32_t lead = h.z, flags = h.w;
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll 1
  for (int u = 0; u < kRows; ++u) {
    const int off = u * kThreads + threadIdx.x;
    const uint32_t word = s_bits[off >> 5];
    if (off >= len || (word >> lane & 1u)) continue;
    const uint32_t g = u * kWarps + warp;
    const uint32_t lv_before = s_lv[g] + __popc(word & lt);  // movers in the tile before off
    const uint32_t r = (uint32_t)(base + off) - (lead + lv_before);
    const uint32_t incl = s_cnt[off];
    const uint32_t a = w0 + s_cs[g] + incl;
    const uint32_t pos = r + a;
    if (pos >= (uint32_t)n || a > m) {
      ar::raise_error(err, ar::kErrOverflow);
      continue;
    }
    out_k[pos] = s_k[off];
    out_v[pos] = s_v[off];
    if ((uint32_t)off > lv_before) {
      // an earlier stayer in the tile: the movers counted here lie between its A and ours
      const uint32_t below = lane ? s_cnt[off - 1] : 0u;  // in-warp inclusive sum before
      for (uint32_t i = a - (incl - below); i < a; ++i) {
        const unsigned long long e = mover(i);
        out_k[r + i] = (uint32_t)(e >> 32);
        out_v[r + i] = (uint32_t)e;
      }
    } else {
      // the tile's first stayer: the movers below A that lie above the previous stayer
      const bool has = flags & kHasPrev;
      const uint4 h1 = w.thead[2 * tile + 1];
      const unsigned long long pc = composite(h1.x, h1.y);
      for (uint32_t i = a; i > 0; --i) {
        const unsigned long long e = mover(i - 1);
        if (has && e < pc) break;
        out_k[r + i - 1] = (uint32_t)(e >> 32);
        out_v[r + i - 1] = (uint32_t)e;
      }
    }
  }
  // the movers above every stayer: written by the tile holding the last stayer (tile 0 when
  // there is no stayer)
  if (flags & kTailOwner) {
    const uint32_t from = (flags & kNoStayers) ? 0u : s_end;
    for (uint32_t i = from + threadIdx.x; i < m; i += kThreads) {
      const uint2 e = w.movers[i];
      out_k[(uint32_t)n - m + i] = e.x;
      out_v[(uint32_t)n - m + i] = e.y;
    }
  }
}

}  // namespace ar_resort
