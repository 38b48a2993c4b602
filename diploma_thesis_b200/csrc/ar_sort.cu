// (a8) Stable LSD radix sort, onesweep style (one histogram pass + one pass per digit with
// decoupled look-back).  Replaces cub::DeviceRadixSort::SortPairs on the reference's path
// (Kernels/particleKernelWrappers.cu:419-534, BVHSource/createMortonCodes.cu:183-218).
//
// Pass structure (per digit of 8 bits, or 9 where that saves a pass; ar_sort::make_plan):
//   * each CTA takes the next tile index from an atomic counter, so every earlier tile is
//     already running or finished (look-back always makes progress);
//   * warps rank their items stably: the lanes holding the same digit are found with one
//     ballot per digit bit, or (on request, 8-bit digits) one match.any per item; items are
//     visited in input order: warp w owns a contiguous sub-range, item j of lane l is element
//     j*32 + l;
//   * per digit, the tile count is published, earlier tiles are looked back through (eight
//     status words per round trip) until an inclusive prefix is found, and the tile's own
//     inclusive prefix is published; the keys are staged and the value loads issued before
//     the look-back, so its latency overlaps them;
//   * items are staged in shared memory in (digit, rank) order and written out with
//     consecutive threads, so each digit run is a coalesced write.
// Spin waits are bounded; on timeout the kernel raises kErrTimeout and finishes the pass
// with whatever prefix it has (the result is then garbage, but nothing hangs).
#include <cuda/atomic>
#include <mutex>

#include "ar_internal.cuh"
#include "ar_sort.cuh"

namespace {

constexpr int kThreads = 256;  // histogram kernel
constexpr int kItems = 16;     // keys per thread in a digit pass
// Threads per digit-pass tile: 512 (8192-key tiles: fewer tiles, shorter look-back chains) from
// 2^19 keys on, 256 below (more tiles to spread over the SMs).
inline int pass_threads(long n) { return n >= (1l << 19) ? 512 : 256; }
inline long tile_items(long n) { return (long)pass_threads(n) * kItems; }
constexpr int kRadix = ar_sort::kMaxRadix;  // histogram / status stride per pass
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kValueMask = (1u << 30) - 1;
constexpr long kSpinLimit = 1l << 24;
constexpr long kTestSpinLimit = 4096;  // AR_SORT_TEST_MUTE_FIRST_TILE: give up quickly
constexpr int kLookWindow = 8;  // look-back status words read per round trip

template <class K>
__device__ __forceinline__ uint32_t digit_of(K key, int shift, uint32_t mask) {
  return (uint32_t)(key >> shift) & mask;
}

// ---- histogram of every pass, one read of the keys -----------------------------------------
template <class K>
__global__ void __launch_bounds__(kThreads) hist_kernel(const K* __restrict__ keys, int n,
                                                       ar_sort::Plan plan,
                                                       uint32_t* __restrict__ hist) {
  ar::pdl_wait();
  __shared__ uint32_t s_hist[ar_sort::kMaxPasses][kRadix];
  const int passes = plan.passes;
  for (int i = threadIdx.x; i < passes * kRadix; i += kThreads) (&s_hist[0][0])[i] = 0;
  __syncthreads();
  for (int i = blockIdx.x * kThreads + threadIdx.x; i < n; i += gridDim.x * kThreads) {
    K k = keys[i];
    for (int p = 0; p < passes; ++p)
      atomicAdd(&s_hist[p][digit_of(k, plan.shift[p], (1u << plan.bits[p]) - 1)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * kRadix; i += kThreads) {
    uint32_t v = (&s_hist[0][0])[i];
    if (v) atomicAdd(hist + i, v);
  }
}

// Exclusive scan of each pass's histogram (kRadix bins; one warp per pass).
__global__ void hist_scan_kernel(uint32_t* __restrict__ hist, int passes) {
  ar::pdl_wait();
  int p = threadIdx.x >> 5;
  if (p >= passes) return;
  uint32_t* h = hist + p * kRadix;
  int lane = ar::lane_id();
  uint32_t carry = 0;
  for (int c = 0; c < kRadix; c += 32) {
    uint32_t v = h[c + lane], x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    h[c + lane] = carry + x - v;
    carry += __shfl_sync(0xffffffffu, x, 31);
  }
}

// ---- one digit pass ---------------------------------------------------------------------------
template <class K, int kT, int kBits>
struct PassSmem {
  K keys[kT * kItems];
  uint32_t vals[kT * kItems];
  uint32_t warp_hist[kT / 32][1 << kBits];
  uint32_t digit_start[1 << kBits];  // tile-local exclusive start of each digit
  uint32_t gofs[1 << kBits];         // global destination of the digit's first tile element
  uint32_t tile_id;
};

// One digit pass of at most kBits bits (kBits 9 only with kT 512: one digit per thread).
// kMatch: rank 8-bit digits with one warp match.any per item instead of a ballot per digit
// bit.  Which is faster depends on the keys: match.any wins when a warp's items hold few
// distinct digits (cell keys of particles in input order), ballots win when they hold many
// (Morton codes).
template <class K, int kT, int kBits, bool kMatch = false>
__global__ void __launch_bounds__(kT, (sizeof(K) == 4 ? 1024 : 512) / kT) onesweep_kernel(
    const K* __restrict__ keys_in, const uint32_t* __restrict__ vals_in, K* __restrict__ keys_out,
    uint32_t* __restrict__ vals_out, int n, int shift, int bits,
    const uint32_t* __restrict__ digit_base, uint32_t* __restrict__ status,
    uint32_t* __restrict__ tile_counter, int* __restrict__ err, long spin_limit,
    int mute_tile0) {
  ar::pdl_wait();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int kWarps = kT / 32;
  constexpr int kTile = kT * kItems;
  constexpr int kDigits = 1 << kBits;
  static_assert(kDigits <= kT, "one digit per thread");
  PassSmem<K, kT, kBits>& sm = *reinterpret_cast<PassSmem<K, kT, kBits>*>(smem_raw);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t mask = (1u << bits) - 1;

  if (tid == 0) sm.tile_id = atomicAdd(tile_counter, 1u);
  for (int i = tid; i < kWarps * kDigits; i += kT) (&sm.warp_hist[0][0])[i] = 0;
  __syncthreads();
  const uint32_t tile = sm.tile_id;
  const long tile_base = (long)tile * kTile;

  // load keys (coalesced: item j of lane l in warp w is element base + w*kItems*32 + j*32 + l);
  // values are read only after the keys are staged, and digits are recomputed from the keys,
  // which keeps the register count (and so the occupancy) down
  K key[kItems];
  uint32_t rank[kItems];
  const long wbase = tile_base + (long)warp * kItems * 32;
#pragma unroll
  for (int j = 0; j < kItems; ++j) {
    long g = wbase + j * 32 + lane;
    // invalid items take digit kDigits-1 (after every valid item of the tile; never written)
    key[j] = g < n ? keys_in[g] : (K)~(K)0;
  }

  // stable warp multi-split: peers = lanes holding the same digit
  const uint32_t lt = (1u << lane) - 1;
#pragma unroll
  for (int j = 0; j < kItems; ++j) {
    const long g = wbase + j * 32 + lane;
    const uint32_t dj = g < n ? digit_of(key[j], shift, mask) : kDigits - 1;
    uint32_t peers;
    if constexpr (kMatch && kBits <= 8) {
      peers = __match_any_sync(0xffffffffu, dj);
    } else {
      peers = 0xffffffffu;
      for (int b = 0; b < kBits; ++b) {
        const uint32_t bit = (dj >> b) & 1u;
        const uint32_t m = __ballot_sync(0xffffffffu, bit);
        peers &= bit ? m : ~m;
      }
    }
    uint32_t before = __popc(peers & lt);
    int leader = __ffs(peers) - 1;
    __syncwarp();
    uint32_t old = sm.warp_hist[warp][dj];
    __syncwarp();
    if (lane == leader) sm.warp_hist[warp][dj] = old + __popc(peers);
    rank[j] = old + before;
  }
  __syncthreads();

  // per digit: exclusive over warps, tile count; the tile's aggregate is published at once
  const int d = tid;  // threads below kDigits own one digit each
  uint32_t tile_count = 0;
  if (d < kDigits) {
#pragma unroll
    for (int w = 0; w < kWarps; ++w) {
      uint32_t c = sm.warp_hist[w][d];
      sm.warp_hist[w][d] = tile_count;
      tile_count += c;
    }
    cuda::atomic_ref<uint32_t, cuda::thread_scope_device> mine(status[(long)tile * kRadix + d]);
    if (!(mute_tile0 && tile == 0))
      mine.store((tile == 0 ? kFlagPrefix : kFlagAgg) | tile_count, cuda::memory_order_relaxed);
  }

  // tile-local exclusive scan over digits (block scan of one value per thread)
  {
    uint32_t x = tile_count;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    __shared__ uint32_t s_wsum[kWarps];
    if (lane == 31) s_wsum[warp] = x;
    __syncthreads();
    uint32_t add = 0;
    for (int w = 0; w < warp; ++w) add += s_wsum[w];
    if (d < kDigits) sm.digit_start[d] = add + x - tile_count;
  }
  __syncthreads();

  // stage the keys in (digit, rank) order (rank[] becomes the staging slot), then start the
  // value loads so that they are in flight during the look-back
#pragma unroll
  for (int j = 0; j < kItems; ++j) {
    const long g = wbase + j * 32 + lane;
    if (g < n) {
      const uint32_t dj = digit_of(key[j], shift, mask);
      rank[j] += sm.digit_start[dj] + sm.warp_hist[warp][dj];
      sm.keys[rank[j]] = key[j];
    }
  }
  uint32_t val[kItems];
#pragma unroll
  for (int j = 0; j < kItems; ++j) {
    const long g = wbase + j * 32 + lane;
    val[j] = g < n ? (vals_in ? __ldg(vals_in + g) : (uint32_t)g) : 0u;
  }

  // look back through the earlier tiles, kLookWindow status words per round trip, until an
  // inclusive prefix is found; then publish this tile's inclusive prefix
  if (d < kDigits) {
    uint32_t excl = 0;
    if (tile != 0) {
      long k = (long)tile - 1;  // next tile to read
      long spins = 0;
      bool found = false;
      while (!found) {
        uint32_t v[kLookWindow];
#pragma unroll
        for (int w = 0; w < kLookWindow; ++w) {
          v[w] = kFlagPrefix;  // before tile 0: never reached (tile 0 is inclusive)
          if (k - w >= 0) {
            cuda::atomic_ref<uint32_t, cuda::thread_scope_device> other(
                status[(k - w) * kRadix + d]);
            v[w] = other.load(cuda::memory_order_relaxed);
          }
        }
        int used = 0;
#pragma unroll
        for (int w = 0; w < kLookWindow; ++w) {
          const uint32_t flag = v[w] & ~kValueMask;
          if (flag == 0) break;  // not published yet: read again from this tile
          excl += v[w] & kValueMask;
          ++used;
          if (flag == kFlagPrefix) {
            found = true;
            break;
          }
        }
        k -= used;
        if (!found && used == 0) {
          if (++spins > spin_limit) {
            ar::raise_error(err, ar::kErrTimeout);
            break;
          }
          if (spins > 64) __nanosleep(64);
        }
      }
      cuda::atomic_ref<uint32_t, cuda::thread_scope_device> mine(status[(long)tile * kRadix + d]);
      mine.store(kFlagPrefix | ((excl + tile_count) & kValueMask), cuda::memory_order_relaxed);
    }
    sm.gofs[d] = digit_base[d] + excl;
  }

#pragma unroll
  for (int j = 0; j < kItems; ++j) {
    const long g = wbase + j * 32 + lane;
    if (g < n) sm.vals[rank[j]] = val[j];
  }
  __syncthreads();

  // coalesced write-out
  long valid = n - tile_base;
  int count = valid < kTile ? (int)valid : kTile;
  for (int i = tid; i < count; i += kT) {
    K k = sm.keys[i];
    uint32_t dd = digit_of(k, shift, mask);
    uint32_t dst = sm.gofs[dd] + (uint32_t)i - sm.digit_start[dd];
    if (dst >= (uint32_t)n) {  // only after a timed-out look-back; never write out of range
      ar::raise_error(err, ar::kErrTimeout);
      continue;
    }
    keys_out[dst] = k;
    vals_out[dst] = sm.vals[i];
  }
}

// How the digit passes run: ranking by match.any (8-bit digits), the look-back's spin limit,
// and the failure-detection hook that keeps tile 0 from publishing its status (every later
// tile's look-back then runs out of spins, reports kErrTimeout and writes nothing out of
// range).
struct PassOpts {
  bool match_rank = false;
  long spin_limit = kSpinLimit;
  int mute_tile0 = 0;
};

// The digit passes of `plan`, ping-ponging so that the last one lands in keys_out.  `status`
// holds one [tiles][kRadix] block per pass, tiles = the most tiles any pass uses.
template <class K>
void launch_passes(const ar_sort::Plan& plan, int n, const K* keys_in, const uint32_t* vals_in,
                   K* keys_out, uint32_t* vals_out, K* tmp_keys, uint32_t* tmp_vals,
                   const uint32_t* hist, uint32_t* status, uint32_t* counters, int* err,
                   cudaStream_t st, const PassOpts& o) {
  const long status_tiles = ((long)n + tile_items(n) - 1) / tile_items(n);
  const K* src_k = keys_in;
  const uint32_t* src_v = vals_in;
  for (int p = 0; p < plan.passes; ++p) {
    const bool to_out = ((plan.passes - 1 - p) % 2) == 0;
    K* dk = to_out ? keys_out : tmp_keys;
    uint32_t* dv = to_out ? vals_out : tmp_vals;
    const int bits = plan.bits[p], shift = plan.shift[p];
    const int kt = bits > 8 ? 512 : pass_threads(n);
    const unsigned tiles = (unsigned)(((long)n + (long)kt * kItems - 1) / ((long)kt * kItems));
    const uint32_t* base = hist + p * kRadix;
    uint32_t* stat = status + (size_t)p * status_tiles * kRadix;
    if (bits > 8)
      arh::launch_pdl(onesweep_kernel<K, 512, 9>, dim3(tiles), dim3(512),
          sizeof(PassSmem<K, 512, 9>), st, src_k, src_v, dk, dv, n, shift, bits, base, stat,
          counters + p, err, o.spin_limit, o.mute_tile0);
    else if (kt == 512)
      arh::launch_pdl(o.match_rank ? onesweep_kernel<K, 512, 8, true> : onesweep_kernel<K, 512, 8>,
          dim3(tiles), dim3(512), sizeof(PassSmem<K, 512, 8>), st, src_k, src_v, dk, dv, n, shift,
          bits, base, stat, counters + p, err, o.spin_limit, o.mute_tile0);
    else
      arh::launch_pdl(o.match_rank ? onesweep_kernel<K, 256, 8, true> : onesweep_kernel<K, 256, 8>,
          dim3(tiles), dim3(256), sizeof(PassSmem<K, 256, 8>), st, src_k, src_v, dk, dv, n, shift,
          bits, base, stat, counters + p, err, o.spin_limit, o.mute_tile0);
    src_k = dk;
    src_v = dv;
  }
}

// external_hist: the caller already cleared the workspace head (ar_sort::clear_bytes) and
// accumulated the per-pass histograms into it (ar_sort::hist_count_warp + hist_flush), e.g.
// fused into the kernel that produced the keys.
template <class K>
ar_status sort_impl(ar_ctx* ctx, const K* keys_in, const uint32_t* vals_in, K* keys_out,
                    uint32_t* vals_out, int n, int begin_bit, int end_bit, cudaStream_t st,
                    void* ws, size_t ws_bytes, bool external_hist = false,
                    const PassOpts& opts = PassOpts()) {
  const ar_sort::Plan plan = ar_sort::make_plan(begin_bit, end_bit);
  const int passes = plan.passes;
  ar_sort::Layout L = ar_sort::layout(n, sizeof(K), passes);
  if (ws_bytes < L.total) {
    arh::set_error("radix sort: workspace too small");
    return AR_ERR_INVALID_ARG;
  }
  char* base = (char*)ws;
  uint32_t* hist = (uint32_t*)(base + L.hist);
  uint32_t* counters = (uint32_t*)(base + L.counters);
  uint32_t* status = (uint32_t*)(base + L.status);
  K* tmp_keys = (K*)(base + L.tmp_keys);
  uint32_t* tmp_vals = (uint32_t*)(base + L.tmp_vals);
  int* err = ctx ? ctx->d_err : nullptr;

  if (!external_hist) {
    cudaMemsetAsync(base, 0, ar_sort::clear_bytes(n, passes), st);
    unsigned hgrid = (unsigned)((n + kThreads * 8 - 1) / (kThreads * 8));
    unsigned cap = (unsigned)(ctx ? ctx->num_sms : 148) * 4;
    if (hgrid > cap) hgrid = cap;
    if (hgrid < 1) hgrid = 1;
    arh::launch_pdl(hist_kernel<K>, dim3(hgrid), dim3(kThreads), 0, st, keys_in, n, plan, hist);
  }
  arh::launch_pdl(hist_scan_kernel, dim3(1), dim3(32 * ar_sort::kMaxPasses), 0, st, hist, passes);
  launch_passes<K>(plan, n, keys_in, vals_in, keys_out, vals_out, tmp_keys, tmp_vals, hist,
                   status, counters, err, st, opts);
  return arh::check_launch("radix sort");
}

// True when the byte ranges [a, a + a_bytes) and [b, b + b_bytes) share any byte.
inline bool overlaps(const void* a, size_t a_bytes, const void* b, size_t b_bytes) {
  const uintptr_t x = (uintptr_t)a, y = (uintptr_t)b;
  return x < y + b_bytes && y < x + a_bytes;
}

// Argument checks shared by every sort entry point (n > 0): an output that overlaps its input
// anywhere would be overwritten by the first pass while other tiles still read it.
template <class K>
ar_status check_sort_args(const K* keys_in, const uint32_t* vals_in, const K* keys_out,
                          const uint32_t* vals_out, int n, const char* who) {
  if (!keys_in || !keys_out || !vals_out) return AR_ERR_INVALID_ARG;
  const size_t kb = (size_t)n * sizeof(K), vb = (size_t)n * 4;
  if (overlaps(keys_in, kb, keys_out, kb) || overlaps(keys_in, kb, vals_out, vb) ||
      (vals_in && (overlaps(vals_in, vb, vals_out, vb) || overlaps(vals_in, vb, keys_out, kb))) ||
      overlaps(keys_out, kb, vals_out, vb)) {
    arh::set_error("%s: outputs must not overlap the inputs or each other", who);
    return AR_ERR_INVALID_ARG;
  }
  return AR_OK;
}

template <class K>
ar_status sort_entry(ar_ctx* ctx, const K* keys_in, const uint32_t* vals_in, K* keys_out,
                     uint32_t* vals_out, int n, int begin_bit, int end_bit, ar_stream_t stream,
                     const PassOpts& opts = PassOpts()) {
  const int kbits = 8 * (int)sizeof(K);
  if (!ctx || n < 0 || begin_bit < 0 || end_bit > kbits || begin_bit > end_bit)
    return AR_ERR_INVALID_ARG;
  if (n > 0) {
    const ar_status a = check_sort_args(keys_in, vals_in, keys_out, vals_out, n, "radix sort");
    if (a != AR_OK) return a;
  }
  if (n >= (1 << 30)) {
    arh::set_error("radix sort: n must be < 2^30");
    return AR_ERR_INVALID_ARG;
  }
  cudaStream_t st = arh::stream(stream);
  if (n == 0) return AR_OK;
  if (begin_bit == end_bit) {  // nothing to sort: copy through
    cudaMemcpyAsync(keys_out, keys_in, (size_t)n * sizeof(K), cudaMemcpyDeviceToDevice, st);
    if (vals_in)
      cudaMemcpyAsync(vals_out, vals_in, (size_t)n * 4, cudaMemcpyDeviceToDevice, st);
    else
      ar_sort::iota(vals_out, n, st);
    return arh::check_launch("radix sort copy");
  }
  const int passes = ar_sort::make_plan(begin_bit, end_bit).passes;
  ar_sort::Layout L = ar_sort::layout(n, sizeof(K), passes);
  void* ws = arh::scratch(ctx, L.total);
  if (!ws) return AR_ERR_OOM;
  return sort_impl<K>(ctx, keys_in, vals_in, keys_out, vals_out, n, begin_bit, end_bit, st, ws,
                      L.total, false, opts);
}

__global__ void iota_kernel(uint32_t* v, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] = i;
}

// Dynamic shared-memory opt-in of every digit-pass instantiation (current device).
template <class K, int kT, int kBits, bool kMatch = false>
cudaError_t set_pass_attribute() {
  return cudaFuncSetAttribute(onesweep_kernel<K, kT, kBits, kMatch>,
                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)sizeof(PassSmem<K, kT, kBits>));
}
cudaError_t set_pass_attributes() {
  cudaError_t e = set_pass_attribute<uint32_t, 256, 8>();
  if (e == cudaSuccess) e = set_pass_attribute<uint32_t, 512, 8>();
  if (e == cudaSuccess) e = set_pass_attribute<uint32_t, 512, 9>();
  if (e == cudaSuccess) e = set_pass_attribute<uint32_t, 256, 8, true>();
  if (e == cudaSuccess) e = set_pass_attribute<uint32_t, 512, 8, true>();
  if (e == cudaSuccess) e = set_pass_attribute<uint64_t, 256, 8>();
  if (e == cudaSuccess) e = set_pass_attribute<uint64_t, 512, 8>();
  if (e == cudaSuccess) e = set_pass_attribute<uint64_t, 512, 9>();
  return e;
}

// ---- allocation-free variant -------------------------------------------------------------------
// Workspace of the u32 sort for up to kNoAllocMaxN pairs, laid out like ar_sort::layout
// (histograms, tile counters, look-back status for 4 passes, ping-pong keys and values).
constexpr int kNoAllocMaxN = 1 << 20;
constexpr size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t noalloc_bytes() {
  return up256(up256(up256(up256(up256((size_t)ar_sort::kMaxPasses * kRadix * 4) +
                                       ar_sort::kMaxPasses * 4) +
                                 (size_t)4 * (kNoAllocMaxN / (256 * kItems)) * kRadix * 4) +
                           (size_t)kNoAllocMaxN * 4) +
               (size_t)kNoAllocMaxN * 4);
}
// One copy per GPU that loads the library, held until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[noalloc_bytes()];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_addr[kNoAllocMaxDevices] = {};
int g_noalloc_sms[kNoAllocMaxDevices] = {};

// Per-device set-up, once, with that device current: the device address of the static
// workspace (host code cannot use the symbol's name as an address) and the shared-memory
// opt-in of the pass kernel.
ar_status noalloc_setup(int dev, void** addr, int* sms) {
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      arh::set_error("allocation-free sort: cudaGetSymbolAddress failed (%s)",
                     cudaGetErrorString(e));
      return AR_ERR_CUDA;
    }
    e = set_pass_attributes();
    if (e != cudaSuccess) {
      arh::set_error("allocation-free sort: %s", cudaGetErrorString(e));
      return AR_ERR_CUDA;
    }
    int n_sms = 148;
    cudaDeviceGetAttribute(&n_sms, cudaDevAttrMultiProcessorCount, dev);
    g_noalloc_sms[dev] = n_sms;
    g_noalloc_addr[dev] = p;
  }
  *addr = g_noalloc_addr[dev];
  *sms = g_noalloc_sms[dev];
  return AR_OK;
}

}  // namespace

namespace ar_sort {

void init() { set_pass_attributes(); }

Layout layout(long n, size_t key_bytes, int passes) {
  const long tiles = (n + tile_items(n) - 1) / tile_items(n);
  auto up = [](size_t x) { return (x + 255) & ~(size_t)255; };
  Layout L;
  L.hist = 0;
  L.counters = up(L.hist + (size_t)kMaxPasses * kRadix * 4);
  L.status = up(L.counters + kMaxPasses * 4);
  L.tmp_keys = up(L.status + (size_t)passes * tiles * kRadix * 4);
  L.tmp_vals = up(L.tmp_keys + (size_t)n * key_bytes);
  L.total = up(L.tmp_vals + (size_t)n * 4);
  return L;
}

void iota(uint32_t* v, int n, cudaStream_t st) {
  iota_kernel<<<arh::grid_for(n, 256) > 4096 ? 4096 : arh::grid_for(n, 256), 256, 0, st>>>(v, n);
}

ar_status sort_u32(ar_ctx* ctx, const uint32_t* keys_in, const uint32_t* vals_in,
                   uint32_t* keys_out, uint32_t* vals_out, int n, int begin_bit, int end_bit,
                   cudaStream_t st, void* ws, size_t ws_bytes, bool external_hist,
                   bool match_rank) {
  if (n == 0) return AR_OK;
  PassOpts o;
  o.match_rank = match_rank;
  return sort_impl<uint32_t>(ctx, keys_in, vals_in, keys_out, vals_out, n, begin_bit, end_bit,
                             st, ws, ws_bytes, external_hist, o);
}

ar_status sort_u64(ar_ctx* ctx, const uint64_t* keys_in, const uint32_t* vals_in,
                   uint64_t* keys_out, uint32_t* vals_out, int n, int begin_bit, int end_bit,
                   cudaStream_t st, void* ws, size_t ws_bytes) {
  if (n == 0) return AR_OK;
  return sort_impl<uint64_t>(ctx, keys_in, vals_in, keys_out, vals_out, n, begin_bit, end_bit,
                             st, ws, ws_bytes, false);
}

size_t clear_bytes(long n, int passes) {
  const long tiles = (n + tile_items(n) - 1) / tile_items(n);
  Layout L = layout(n, 4, passes);
  return L.status + (size_t)passes * tiles * kRadix * sizeof(uint32_t);
}

int launches(int begin_bit, int end_bit, bool external_hist) {
  return (external_hist ? 1 : 3) + make_plan(begin_bit, end_bit).passes;
}

}  // namespace ar_sort

extern "C" {

ar_status ar_radix_sort_pairs_u32(ar_ctx* ctx, const uint32_t* keys_in, const uint32_t* vals_in,
                                  uint32_t* keys_out, uint32_t* vals_out, int n, int begin_bit,
                                  int end_bit, ar_stream_t stream) {
  return sort_entry<uint32_t>(ctx, keys_in, vals_in, keys_out, vals_out, n, begin_bit, end_bit,
                              stream);
}

ar_status ar_radix_sort_pairs_u64(ar_ctx* ctx, const uint64_t* keys_in, const uint32_t* vals_in,
                                  uint64_t* keys_out, uint32_t* vals_out, int n, int begin_bit,
                                  int end_bit, ar_stream_t stream) {
  return sort_entry<uint64_t>(ctx, keys_in, vals_in, keys_out, vals_out, n, begin_bit, end_bit,
                              stream);
}

ar_status ar_radix_sort_pairs_u32_ex(ar_ctx* ctx, const uint32_t* keys_in,
                                     const uint32_t* vals_in, uint32_t* keys_out,
                                     uint32_t* vals_out, int n, int begin_bit, int end_bit,
                                     uint32_t flags, ar_stream_t stream) {
  const uint32_t known = AR_SORT_RANK_MATCH | AR_SORT_TEST_MUTE_FIRST_TILE;
  if (flags & ~known) {
    arh::set_error("radix sort: unknown flags 0x%x", flags & ~known);
    return AR_ERR_INVALID_ARG;
  }
  PassOpts o;
  o.match_rank = (flags & AR_SORT_RANK_MATCH) != 0;
  if (flags & AR_SORT_TEST_MUTE_FIRST_TILE) {
    o.mute_tile0 = 1;
    o.spin_limit = kTestSpinLimit;
  }
  return sort_entry<uint32_t>(ctx, keys_in, vals_in, keys_out, vals_out, n, begin_bit, end_bit,
                              stream, o);
}

// The same sort as ar_radix_sort_pairs_u32, with its workspace in g_noalloc_scratch instead
// of memory from cudaMalloc.  Shared by every call on a device: calls that overlap on the
// GPU race; the histogram / look-back head is cleared at the start of each call.
ar_status ar_radix_sort_pairs_u32_noalloc(const uint32_t* keys_in, const uint32_t* vals_in,
                                          uint32_t* keys_out, uint32_t* vals_out, int n,
                                          int begin_bit, int end_bit, int32_t* d_status,
                                          ar_stream_t stream) {
  if (n < 0 || begin_bit < 0 || end_bit > 32 || begin_bit > end_bit) return AR_ERR_INVALID_ARG;
  if (n > kNoAllocMaxN) {
    arh::set_error("allocation-free sort: n = %d exceeds its limit of %d pairs", n, kNoAllocMaxN);
    return AR_ERR_INVALID_ARG;
  }
  if (n > 0) {
    const ar_status a =
        check_sort_args(keys_in, vals_in, keys_out, vals_out, n, "allocation-free sort");
    if (a != AR_OK) return a;
  }
  if (n == 0) return AR_OK;
  cudaStream_t st = arh::stream(stream);
  if (begin_bit == end_bit) {
    cudaMemcpyAsync(keys_out, keys_in, (size_t)n * 4, cudaMemcpyDeviceToDevice, st);
    if (vals_in)
      cudaMemcpyAsync(vals_out, vals_in, (size_t)n * 4, cudaMemcpyDeviceToDevice, st);
    else
      ar_sort::iota(vals_out, n, st);
    return arh::check_launch("allocation-free sort copy");
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) {
    arh::set_error("allocation-free sort: no usable current device");
    return AR_ERR_CUDA;
  }
  void* base_v = nullptr;
  int sms = 148;
  ar_status s = noalloc_setup(dev, &base_v, &sms);
  if (s != AR_OK) return s;
  const ar_sort::Plan plan = ar_sort::make_plan(begin_bit, end_bit);
  const int passes = plan.passes;
  const ar_sort::Layout L = ar_sort::layout(n, 4, passes);
  if (L.total > sizeof(g_noalloc_scratch)) {  // cannot happen for n <= kNoAllocMaxN
    arh::set_error("allocation-free sort: workspace layout exceeds the static array");
    return AR_ERR_INVALID_ARG;
  }
  char* base = (char*)base_v;
  uint32_t* hist = (uint32_t*)(base + L.hist);
  uint32_t* counters = (uint32_t*)(base + L.counters);
  uint32_t* status = (uint32_t*)(base + L.status);
  uint32_t* tmp_keys = (uint32_t*)(base + L.tmp_keys);
  uint32_t* tmp_vals = (uint32_t*)(base + L.tmp_vals);
  // the previous call's contents stay in the array: zero what must start at zero
  cudaMemsetAsync(base, 0, ar_sort::clear_bytes(n, passes), st);
  unsigned hgrid = (unsigned)((n + kThreads * 8 - 1) / (kThreads * 8));
  if (hgrid > (unsigned)sms * 4) hgrid = (unsigned)sms * 4;
  if (hgrid < 1) hgrid = 1;
  arh::launch_pdl(hist_kernel<uint32_t>, dim3(hgrid), dim3(kThreads), 0, st, keys_in, n, plan,
      hist);
  arh::launch_pdl(hist_scan_kernel, dim3(1), dim3(32 * ar_sort::kMaxPasses), 0, st, hist, passes);
  launch_passes<uint32_t>(plan, n, keys_in, vals_in, keys_out, vals_out, tmp_keys, tmp_vals, hist,
                          status, counters, (int*)d_status, st, PassOpts());
  return arh::check_launch("allocation-free sort");
}

}  // extern "C"
