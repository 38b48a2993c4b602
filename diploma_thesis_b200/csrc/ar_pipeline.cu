// Fused PHYSICAL-mode step over a table of resident scenes.
//
// Per step (one launch per stage, whatever the number of scenes):
//   K0       clear the sort's counters and one 255th of the cell table (see cell_epoch)
//   K1       re-pose + hash: key = scene cell base + wrapped cell of the particle's world
//            position
//   sort     the order by (key, global particle index): re-sorted from the last step's order
//            (ar_resort.cuh: particles whose key changed found, bucketed and sorted, every
//            particle placed); the first
//            step after a change of the member list radix-sorts instead (onesweep passes,
//            histogram accumulated in K1)
//   K3       scatter + cell table: sorted position (w = global body id) and velocity,
//            recomputed from the body state; first slot, count, step epoch and body tag of
//            every occupied cell; the order kept for the next step
//   K4       DEM gather over the 27 neighbour cells + box walls -> per-particle force at the
//            particle's original index (no atomics)
//   K5       one warp per body: fixed-order sum of F and r x F; then one thread per body
//            integrates (a separate kernel)
// A scene's keys live in its own cell range, so sorting all scenes together orders them by
// scene and within a scene exactly as a solo sort would: batched and solo steps are
// bit-identical.  The sequence is captured once into a CUDA graph and replayed.
//
// Batches of BVH scenes replace K0-K4 by: a memset of the refit's arrival counters; Morton keys
// (scene index above the particle's 30-bit code: 32-bit keys for up to 4 scenes, else 64-bit);
// the sort (32-bit keys re-sorted from the last step's order as above, 64-bit keys radix-sorted
// every step); Karras nodes over all scenes (equal codes tie-broken by the index within the
// scene); leaves in sorted order, each leaf's thread then climbing the refit (acquire-release
// arrival counters); each scene's subtree root; and per particle a walk of its scene's subtree
// in the reference's visit order with a 64-entry stack.  K5 is shared.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "ar_internal.cuh"
#include "ar_dem.cuh"
#include "ar_lbvh.cuh"
#include "ar_pipeline.cuh"
#include "ar_resort.cuh"
#include "ar_sort.cuh"

using ar_pipe::SceneDev;

namespace {

constexpr int kK1Threads = 256;

__device__ __forceinline__ int find_range(const int* __restrict__ off, int count, int g) {
  int lo = 0, hi = count;  // off[lo] <= g < off[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(off + mid) <= g) lo = mid; else hi = mid;
  }
  return lo;
}

// Cell entry (8 bytes): {first sorted slot, meta}, meta = occupant count (bits 0-4; 31 means
// "31 or more", the end is then found from the sorted keys) | epoch (bits 5-12) | body tag
// (bits 13-31: scene-local body + 1 when every occupant belongs to that body, else 0).
// The epoch is the step number mod 255, plus 1; an entry whose epoch is not the current
// step's reads as empty, so the table is never cleared as a whole.  Instead the first kernel
// of each step zeroes one of 255 slices of the table (slice = step number mod 255), so every
// entry is zeroed within 255 steps of being written, before its epoch can recur; a zero entry
// has epoch 0, which never matches.
constexpr uint32_t kCountMask = 31;
constexpr uint32_t kEpochShift = 5;
constexpr uint32_t kEpochMask = 255;
constexpr uint32_t kTagShift = 13;
constexpr uint32_t kMaxTag = (1u << 19) - 1;  // bodies of a scene with local index + 1 above
                                              // this carry no tag (never skipped)
constexpr int kEpochSlices = 255;
__device__ __forceinline__ uint32_t cell_epoch(long long step) {
  return (uint32_t)(step % kEpochSlices) + 1u;
}
__device__ __forceinline__ uint32_t body_tag(int local_body) {
  return (uint32_t)local_body + 1u <= kMaxTag ? (uint32_t)local_body + 1u : 0u;
}

// The scene of a particle or body.  A batch of one scene passes its descriptor itself as a
// kernel parameter (kOne): it is read from the constant bank, and no lookup of the scene index
// and the table entry sits in front of the particle's own loads.
template <bool kOne>
__device__ __forceinline__ const SceneDev& scene_at(const SceneDev& one,
                                                    const SceneDev* __restrict__ table, int s) {
  if constexpr (kOne) return one;
  else return table[s];
}

// Scene index of every particle and body of the batch (run when the member list changes).
__global__ void __launch_bounds__(256) scene_ids_kernel(const int* __restrict__ poff,
                                                        const int* __restrict__ boff, int ns,
                                                        int nt, int bt, int* __restrict__ pscene,
                                                        int* __restrict__ bscene) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nt || i < bt;
       i += gridDim.x * blockDim.x) {
    if (i < nt) pscene[i] = find_range(poff, ns, i);
    if (i < bt) bscene[i] = find_range(boff, ns, i);
  }
}

// ---- K0: clears ------------------------------------------------------------------------------
// Zeroes the head of the sort about to run (the radix sort's histogram / look-back counters, or
// the re-sort's counters) and the cell-table slice of the step about to run (its number is
// *d_step + 1; K1 increments the counter).
__global__ void __launch_bounds__(256) step_clear_kernel(uint4* __restrict__ head, long head16,
                                                         uint2* __restrict__ cells,
                                                         unsigned long long num_cells,
                                                         const long long* __restrict__ d_step) {
  ar::pdl_wait();
  const long stride = (long)gridDim.x * blockDim.x;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  for (long i = t; i < head16; i += stride) head[i] = make_uint4(0u, 0u, 0u, 0u);
  const unsigned long long len = (num_cells + kEpochSlices - 1) / kEpochSlices;
  const unsigned long long lo = (unsigned long long)((*d_step + 1) % kEpochSlices) * len;
  const unsigned long long hi = lo + len < num_cells ? lo + len : num_cells;
  for (unsigned long long i = lo + t; i < hi; i += stride) cells[i] = make_uint2(0u, 0u);
}

// ---- K1: re-pose + cell keys (+ sort histogram) ---------------------------------------------
// Each thread takes kKeysBatch particles per round (stride apart, so each load is coalesced)
// and issues the loads of all of them before using any, which keeps several dependent
// gathers (scene -> offset -> body) in flight per thread.  kHist: the radix sort's histogram
// is accumulated (a step that re-sorts needs none).
constexpr int kKeysBatch = 2;
template <bool kOne, bool kHist>
__global__ void __launch_bounds__(kK1Threads) grid_keys_kernel(
    const __grid_constant__ SceneDev one, const SceneDev* __restrict__ table,
    const int* __restrict__ pscene, int nt,
    uint32_t* __restrict__ keys, uint32_t* __restrict__ ws_hist, ar_sort::Plan plan,
    long long* __restrict__ d_step) {
  ar::pdl_wait();
  __shared__ uint32_t s_hist[ar_sort::kMaxPasses][ar_sort::kMaxRadix];
  if (blockIdx.x == 0 && threadIdx.x == 0) *d_step += 1;  // this step's number
  if (kHist) {
    for (int i = threadIdx.x; i < plan.passes * ar_sort::kMaxRadix; i += blockDim.x)
      (&s_hist[0][0])[i] = 0;
    __syncthreads();
  }
  const int stride = gridDim.x * blockDim.x;
  for (int g0 = blockIdx.x * blockDim.x + threadIdx.x; g0 < nt; g0 += stride * kKeysBatch) {
    int sc[kKeysBatch];
    float4 r4[kKeysBatch], q[kKeysBatch], c[kKeysBatch];
#pragma unroll
    for (int u = 0; u < kKeysBatch; ++u) {
      const int g = g0 + u * stride;
      sc[u] = !kOne && g < nt ? __ldg(pscene + g) : 0;
    }
#pragma unroll
    for (int u = 0; u < kKeysBatch; ++u) {
      const int g = g0 + u * stride;
      if (g < nt) {
        const SceneDev& S = scene_at<kOne>(one, table, sc[u]);
        r4[u] = __ldg(S.rel + (g - S.poff));
      }
    }
#pragma unroll
    for (int u = 0; u < kKeysBatch; ++u) {
      const int g = g0 + u * stride;
      if (g < nt) {
        const SceneDev& S = scene_at<kOne>(one, table, sc[u]);
        const int b = __float_as_int(r4[u].w);
        q[u] = __ldg(S.quat + b);
        c[u] = __ldg(S.pos + b);
      }
    }
#pragma unroll
    for (int u = 0; u < kKeysBatch; ++u) {
      const int g = g0 + u * stride;
      if (g < nt) {
        const SceneDev& S = scene_at<kOne>(one, table, sc[u]);
        const float3 r = ar::quat_rotate(q[u], ar::mk3(r4[u].x, r4[u].y, r4[u].z));
        const float3 p = ar::add(ar::xyz(c[u]), r);
        const uint32_t key = ar_pipe::cell_key(S, ar_pipe::cell_of(S, p));
        keys[g] = key;
        if (kHist) ar_sort::hist_count_warp(s_hist, key, plan);
      }
    }
  }
  if (kHist) {
    __syncthreads();
    ar_sort::hist_flush(s_hist, ws_hist, plan.passes);
  }
}

// ---- K3: scatter + cell table -------------------------------------------------------------
// One thread per sorted slot k: sorted position (w = global body id) and velocity (w = scene
// index) recomputed from the body state of particle svals[k].  (Gathering by sorted slot is
// faster here than pushing from the original order: scattered 16-byte stores cost more than
// the gathers.)  Cell entry = {first sorted slot, count | epoch | body tag}; the tag names the
// body when every occupant belongs to one body, so that a particle skips a neighbour cell of
// its own body without loading its occupants (they could only be rejected).  The thread at a
// cell's first slot writes the whole entry.  The sorted keys and indices are also copied to
// prev_keys / prev_vals: the order the next step's re-sort starts from.
// kScatterBatch sorted slots per thread and round, loads issued before use (as in K1).
constexpr int kScatterBatch = 1;
template <bool kOne>
__global__ void __launch_bounds__(256) scatter_kernel(
    const __grid_constant__ SceneDev one, const SceneDev* __restrict__ table,
    const int* __restrict__ pscene, int nt,
    const uint32_t* __restrict__ skeys, const uint32_t* __restrict__ svals,
    uint2* __restrict__ cells, float4* __restrict__ spos, float4* __restrict__ svel,
    uint32_t* __restrict__ prev_keys, uint32_t* __restrict__ prev_vals,
    const long long* __restrict__ d_step) {
  ar::pdl_wait();
  const uint32_t epoch = cell_epoch(*d_step) << kEpochShift;
  const int stride = gridDim.x * blockDim.x;
  for (int k0 = blockIdx.x * blockDim.x + threadIdx.x; k0 < nt; k0 += stride * kScatterBatch) {
    uint32_t key[kScatterBatch];
    int g[kScatterBatch], sc[kScatterBatch];
    bool first[kScatterBatch];
    float4 r4[kScatterBatch], q[kScatterBatch], c[kScatterBatch], v[kScatterBatch],
        w[kScatterBatch];
#pragma unroll
    for (int u = 0; u < kScatterBatch; ++u) {
      const int k = k0 + u * stride;
      if (k < nt) {
        key[u] = __ldg(skeys + k);
        g[u] = (int)__ldg(svals + k);
        first[u] = k == 0 || key[u] != __ldg(skeys + k - 1);
        prev_keys[k] = key[u];
        prev_vals[k] = (uint32_t)g[u];
      }
    }
#pragma unroll
    for (int u = 0; u < kScatterBatch; ++u)
      if (k0 + u * stride < nt) sc[u] = kOne ? 0 : __ldg(pscene + g[u]);
#pragma unroll
    for (int u = 0; u < kScatterBatch; ++u) {
      if (k0 + u * stride < nt) {
        const SceneDev& S = scene_at<kOne>(one, table, sc[u]);
        r4[u] = __ldg(S.rel + (g[u] - S.poff));
      }
    }
#pragma unroll
    for (int u = 0; u < kScatterBatch; ++u) {
      if (k0 + u * stride < nt) {
        const SceneDev& S = scene_at<kOne>(one, table, sc[u]);
        const int b = __float_as_int(r4[u].w);
        q[u] = __ldg(S.quat + b);
        c[u] = __ldg(S.pos + b);
        v[u] = __ldg(S.vel + b);
        w[u] = __ldg(S.ang + b);
      }
    }
#pragma unroll
    for (int u = 0; u < kScatterBatch; ++u) {
      const int k = k0 + u * stride;
      if (k >= nt) continue;
      const SceneDev& S = scene_at<kOne>(one, table, sc[u]);
      const int b = __float_as_int(r4[u].w);
      if (first[u]) {
        // occupants of one cell belong to one scene
        uint32_t tag = body_tag(b);
        int e = k + 1;
        for (; e < nt && __ldg(skeys + e) == key[u]; ++e) {
          const int ge = (int)__ldg(svals + e);
          if (__float_as_int(__ldg(S.rel + (ge - S.poff)).w) != b) tag = 0;
        }
        const uint32_t count = (uint32_t)(e - k) < kCountMask ? (uint32_t)(e - k) : kCountMask;
        cells[key[u]] = make_uint2((uint32_t)k, count | epoch | (tag << kTagShift));
      }
      float3 r, p, vv;
      ar_pipe::repose(q[u], c[u], v[u], w[u], ar::mk3(r4[u].x, r4[u].y, r4[u].z), &r, &p, &vv);
      spos[k] = make_float4(p.x, p.y, p.z, __int_as_float(S.boff + b));
      svel[k] = make_float4(vv.x, vv.y, vv.z, __int_as_float(sc[u]));  // w = scene index
    }
  }
}

// ---- K4: DEM gather + walls ----------------------------------------------------------------
// Per sorted particle: the 27 neighbour cells in z, y, x order, occupants in sorted order,
// skipping its own body (itself included); per-cell partial sums added to the total (the order
// of FindAndHandleRigidBodyCollisionsUniformGridKernel, RigidBodies/UniformGridDEM.cu:166-193).
// The particle's cell comes from its sorted key and its scene from the sorted velocity's w.
// The three cells of an x-row are walked as one flattened loop (candidate t of the row maps to
// cell a, b or c and to that cell's partial sum), so a warp's lanes stay in step across cells;
// cells that hold only this particle's body are skipped from their tag without loading their
// occupants, which could only be rejected.  Candidates at squared distance >= the float just
// above (2r)^2 are rejected without the square root: for them sqrtf(d2) >= 2r exactly, so the
// contact test is unchanged.
struct RowCells {
  uint2 a, b, c;
};

template <bool kOne>
__global__ void __launch_bounds__(256, 4) collide_kernel(
    const __grid_constant__ SceneDev one, const SceneDev* __restrict__ table, int nt, const uint32_t* __restrict__ skeys,
    const uint32_t* __restrict__ svals, const uint2* __restrict__ cells,
    const float4* __restrict__ spos, const float4* __restrict__ svel,
    float4* __restrict__ pforce, const long long* __restrict__ d_step) {
  ar::pdl_wait();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nt) return;
  const uint32_t epoch = cell_epoch(*d_step);
  const float4 p4 = __ldg(spos + k);
  const float4 v4 = __ldg(svel + k);
  const SceneDev& S = scene_at<kOne>(one, table, kOne ? 0 : __float_as_int(v4.w));
  const float3 pos = ar::xyz(p4), vel = ar::xyz(v4);
  const int body = __float_as_int(p4.w);
  // the meta word of a cell holding only this body, count bits cleared (an impossible word
  // when the body has no tag)
  const uint32_t btag = body_tag(body - S.boff);
  const uint32_t own = btag ? (epoch << kEpochShift) | (btag << kTagShift) : 0xffffffffu;
  const float thr = 2.0f * S.r;
  const float thr2_up = nextafterf(thr * thr, INFINITY);
  const float kk = S.k, dmp = S.damping, shr = S.shear, att = S.attraction;
  const uint32_t lx = S.lx, ly = S.ly, mx = S.gx - 1, my = S.gy - 1, mz = S.gz - 1;
  const uint32_t base = S.cell_base, local = __ldg(skeys + k) - base;
  const uint32_t x = local & mx, y = (local >> lx) & my, z = local >> (lx + ly);
  const uint32_t xa = (x - 1) & mx, xc = (x + 1) & mx;
  auto row_base = [&](int r) {  // r = 3 (dz + 1) + (dy + 1)
    const uint32_t zz = (z + (uint32_t)(r / 3) - 1u) & mz, yy = (y + (uint32_t)(r % 3) - 1u) & my;
    return base + (zz << (lx + ly)) + (yy << lx);
  };
  // a cell has occupants to visit unless it is empty (another step's entry) or holds only this
  // particle's body
  auto live = [&](uint32_t m) {
    m &= ~kCountMask;
    return ((m >> kEpochShift) & kEpochMask) == epoch && m != own ? 1u : 0u;
  };
  // pass 1: the meta words of all 27 cells (independent loads, all in flight together) ->
  // bit 3 r + i set when cell i (x-1, x, x+1) of row r has occupants to visit
  const uint32_t* __restrict__ meta = reinterpret_cast<const uint32_t*>(cells) + 1;
  uint32_t todo = 0;
#pragma unroll
  for (int r = 0; r < 9; ++r) {
    const size_t rb = row_base(r);
    const uint32_t ma = __ldg(meta + 2 * (rb + xa)), mb = __ldg(meta + 2 * (rb + x)),
                   mc = __ldg(meta + 2 * (rb + xc));
    todo |= (live(ma) | (live(mb) << 1) | (live(mc) << 2)) << (3 * r);
  }
  // pass 2: rows with occupants to visit, in order.  A row without any would add +0 to every
  // component of the total, which leaves it unchanged (the total starts at +0, and a float sum
  // is -0 only when both addends are), so such rows are skipped.
  auto visits = [&](const uint2& c, uint32_t cell) {  // a saturated count is resolved from the keys
    if (!live(c.y)) return 0u;
    uint32_t n = c.y & kCountMask;
    if (n == kCountMask)
      while (c.x + n < (uint32_t)nt && __ldg(skeys + c.x + n) == cell) ++n;
    return n;
  };
  float3 lin = ar::mk3(0.f, 0.f, 0.f);
  while (todo) {
    const int r = (__ffs(todo) - 1) / 3;
    todo &= ~(7u << (3 * r));
    const uint32_t row = row_base(r);
    const RowCells cur{__ldg(cells + row + xa), __ldg(cells + row + x), __ldg(cells + row + xc)};
    const uint32_t na = visits(cur.a, row + xa), nb = visits(cur.b, row + x),
                   nc = visits(cur.c, row + xc);
    const uint32_t nab = na + nb, total = nab + nc;
    float3 fa = ar::mk3(0.f, 0.f, 0.f), fb = fa, fc = fa;
    for (uint32_t t = 0; t < total; ++t) {
      const uint32_t j = t < na ? cur.a.x + t : (t < nab ? cur.b.x + (t - na) : cur.c.x + (t - nab));
      const float4 q4 = __ldg(spos + j);
      if (__float_as_int(q4.w) == body) continue;
      const float3 rp = ar::sub(ar::xyz(q4), pos);
      const float d2 = ar::dot(rp, rp);
      if (!(d2 < thr2_up)) continue;
      const float dist = sqrtf(d2);
      if (!(dist < thr)) continue;
      const float3 v2 = ar::xyz(__ldg(svel + j));
      const float3 f = ar_dem::spring_force(rp, dist, ar::sub(v2, vel), thr, kk, dmp, shr, att);
      if (t < na) fa = ar::add(fa, f);
      else if (t < nab) fb = ar::add(fb, f);
      else fc = ar::add(fc, f);
    }
    lin = ar::add(lin, fa);
    lin = ar::add(lin, fb);
    lin = ar::add(lin, fc);
  }
  lin = ar::add(lin, ar_pipe::wall_force(S, pos, vel));
  pforce[__ldg(svals + k)] = make_float4(lin.x, lin.y, lin.z, 0.f);
}

// ---- K4b: the static point cloud of the scene ---------------------------------------------
// updateUniformGridDEM's simulateAR branch (RigidBodies/UniformGridUpdate.cpp:967-969,
// Find_And_Handle_Augmented_Reality_Collisions_Uniform_Grid_DEM :881-936): after the particle
// contacts and the walls, each particle of a scene with a point cloud takes the impulses of the
// cloud's points within 2r -- the 27 neighbour cells of its own grid in z, y, x order, the
// points of a cell in the cloud's sorted order, per-cell partial sums added to the cloud total
// (FindAndHandleAugmentedRealityCollisionsUniformGridKernel, RigidBodies/UniformGridDEM.cu:
// 301-377) -- and the cloud total is added to its force, as the reference adds it to
// pLinearImpulse.  Launched only when a scene of the batch has a cloud.
template <bool kOne>
__global__ void __launch_bounds__(128) cloud_collide_kernel(
    const __grid_constant__ SceneDev one, const SceneDev* __restrict__ table, int nt,
    const uint32_t* __restrict__ skeys, const uint32_t* __restrict__ svals,
    const float4* __restrict__ spos, const float4* __restrict__ svel,
    float4* __restrict__ pforce) {
  ar::pdl_wait();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nt) return;
  const float4 v4 = __ldg(svel + k);
  const SceneDev& S = scene_at<kOne>(one, table, kOne ? 0 : __float_as_int(v4.w));
  const uint2* __restrict__ cc = S.cloud_cells;
  if (!cc) return;
  const float4* __restrict__ cp = S.cloud_pos;
  const float4* __restrict__ cn = S.cloud_norm;
  const float3 pos = ar::xyz(__ldg(spos + k)), vel = ar::xyz(v4);
  const float thr = 2.0f * S.r;
  const uint32_t lx = S.lx, ly = S.ly, mx = S.gx - 1, my = S.gy - 1, mz = S.gz - 1;
  const uint32_t local = __ldg(skeys + k) - S.cell_base;
  const uint32_t x = local & mx, y = (local >> lx) & my, z = local >> (lx + ly);
  float3 total = ar::mk3(0.f, 0.f, 0.f);
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy) {
      const uint32_t zz = (z + (uint32_t)dz) & mz, yy = (y + (uint32_t)dy) & my;
      const uint32_t row = (zz << (lx + ly)) + (yy << lx);
      for (int dx = -1; dx <= 1; ++dx) {
        const uint2 c = __ldg(cc + row + ((x + (uint32_t)dx) & mx));
        float3 cf = ar::mk3(0.f, 0.f, 0.f);
        for (uint32_t j = c.x; j < c.y; ++j) {
          const float3 rp = ar::sub(ar::xyz(__ldg(cp + j)), pos);
          const float dist = sqrtf(ar::dot(rp, rp));
          if (!(dist < thr)) continue;
          cf = ar::add(cf, ar_dem::scene_force(rp, dist, vel, ar::xyz(__ldg(cn + j)), thr, S.k,
                                               S.damping, S.shear, S.attraction));
        }
        total = ar::add(total, cf);
      }
    }
  float4* f = pforce + __ldg(svals + k);
  const float4 f0 = *f;
  *f = make_float4(f0.x + total.x, f0.y + total.y, f0.z + total.z, f0.w);
}

// Cell key of each cloud point in its scene's grid (cell_base 0).
__global__ void cloud_keys_kernel(SceneDev d, const float4* __restrict__ pos, int m,
                                  uint32_t* __restrict__ keys) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) keys[i] = ar_pipe::cell_key(d, ar_pipe::cell_of(d, ar::xyz(__ldg(pos + i))));
}

// Cloud points and normals in sorted order, and each occupied cell's {first, end}.
__global__ void cloud_place_kernel(const float4* __restrict__ pos, const float4* __restrict__ nrm,
                                   const uint32_t* __restrict__ skeys,
                                   const uint32_t* __restrict__ sidx, int m,
                                   float4* __restrict__ out_pos, float4* __restrict__ out_nrm,
                                   uint2* __restrict__ cells) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  const uint32_t i = __ldg(sidx + k), key = __ldg(skeys + k);
  out_pos[k] = __ldg(pos + i);
  out_nrm[k] = __ldg(nrm + i);
  uint32_t* c = reinterpret_cast<uint32_t*>(cells + key);
  if (k == 0 || __ldg(skeys + k - 1) != key) c[0] = (uint32_t)k;
  if (k == m - 1 || __ldg(skeys + k + 1) != key) c[1] = (uint32_t)k + 1;
}

// ---- BVH broad phase ---------------------------------------------------------------------------
// Key = scene index above a 30-bit Morton code of the particle's world position normalised to
// its scene's box (generateMortonCodes, BVHSource/BVHkernels.cu:646-716).  Sorting all scenes
// together keeps each scene's leaves contiguous, and since no other scene shares its prefix,
// each scene's leaves are one subtree of the Karras tree; equal codes are tie-broken by the
// index within the scene, so that subtree is the one the scene alone would get.
constexpr int kMortonBits = 30;

__device__ __forceinline__ uint32_t spread10(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

__device__ __forceinline__ uint64_t morton_key(const SceneDev& S, int s, float3 p) {
  const float x = (p.x - S.bmin[0]) / (S.bmax[0] - S.bmin[0]);
  const float y = (p.y - S.bmin[1]) / (S.bmax[1] - S.bmin[1]);
  const float z = (p.z - S.bmin[2]) / (S.bmax[2] - S.bmin[2]);
  const uint32_t code = (spread10((uint32_t)fminf(fmaxf(x * 1024.0f, 0.0f), 1023.0f)) << 2) |
                        (spread10((uint32_t)fminf(fmaxf(y * 1024.0f, 0.0f), 1023.0f)) << 1) |
                        spread10((uint32_t)fminf(fmaxf(z * 1024.0f, 0.0f), 1023.0f));
  return ((uint64_t)s << kMortonBits) | code;
}

template <class K, bool kOne>
__global__ void __launch_bounds__(256) morton_key_kernel(const __grid_constant__ SceneDev one,
                                                         const SceneDev* __restrict__ table,
                                                         const int* __restrict__ pscene, int ns,
                                                         int nt, K* __restrict__ keys,
                                                         long long* __restrict__ d_step) {
  ar::pdl_wait();
  if (blockIdx.x == 0 && threadIdx.x == 0) *d_step += 1;  // this step's number
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < nt; g += gridDim.x * blockDim.x) {
    const int s = kOne ? 0 : __ldg(pscene + g);
    const SceneDev& S = scene_at<kOne>(one, table, s);
    const float4 r4 = __ldg(S.rel + (g - S.poff));
    const int b = __float_as_int(r4.w);
    const float3 r = ar::quat_rotate(__ldg(S.quat + b), ar::mk3(r4.x, r4.y, r4.z));
    const float3 p = ar::add(ar::xyz(__ldg(S.pos + b)), r);
    keys[g] = (K)morton_key(S, s, p);
  }
}

// Internal node i (global id n + i) of the fused BVH holds both children's boxes, ids and body
// tags, so one 64-byte fetch decides a traversal step:
//   c[0] = left box (lo.x, lo.y, lo.z, hi.x)    c[1] = (hi.y, hi.z, left id, left tag)
//   c[2] = right box (lo.x, lo.y, lo.z, hi.x)   c[3] = (hi.y, hi.z, right id, right tag)
// Ids < n are leaves (sorted particle slots).  A child's tag is the global body id when every
// leaf below it belongs to that body, else -1: a particle skips a child that holds only its
// own body's particles without descending (they could only be rejected), which leaves the
// order of everything it does visit unchanged.
struct __align__(64) WideNode {
  float4 c[4];
};

__device__ __forceinline__ int* node_ints(WideNode* nodes, int internal) {
  return reinterpret_cast<int*>(nodes + internal);
}
// Box, id and body tag of child `side` (0 left, 1 right) into the parent's slot.
__device__ __forceinline__ void put_child(WideNode* nodes, int internal, int side, float4 lo,
                                          float2 hi_yz, int id, int tag) {
  float4* c = nodes[internal].c + 2 * side;
  __stcg(c, lo);
  __stcg(c + 1, make_float4(hi_yz.x, hi_yz.y, __int_as_float(id), __int_as_float(tag)));
}

template <class Lcp>
__global__ void __launch_bounds__(256) bvh_build_kernel(Lcp lcp, int n,
                                                        uint8_t* __restrict__ is_leaf,
                                                        int32_t* __restrict__ left,
                                                        int32_t* __restrict__ right,
                                                        int32_t* __restrict__ parent,
                                                        int32_t* __restrict__ min_r,
                                                        int32_t* __restrict__ max_r,
                                                        WideNode* __restrict__ nodes) {
  ar::pdl_wait();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) parent[n] = -1;
  if (i >= n - 1) return;
  ar_lbvh::karras_node(i, n, lcp, is_leaf, left, right, parent, min_r, max_r);
}

// Bottom-up refit (kernelConstructInternalNodesSoA, BVHSource/BVHSoAKernels.cu:148-176) from
// one leaf whose box is already in its parent's slot (ar_lbvh::refit_climb): the second thread
// to reach a node merges the two child boxes held in the node (mergeBounds,
// BVHAuxiliary.cuh:83-94) and stores the result, with the merged body tag, into the node's slot
// in its parent, then climbs on.  Release / acquire through the arrival counter; boxes through
// L2.
__device__ __forceinline__ void refit_from_leaf(int i, int n, const int32_t* __restrict__ left,
                                                const int32_t* __restrict__ parent,
                                                WideNode* nodes, int* __restrict__ counters) {
  // The climb of ar_lbvh::refit_climb with the wide nodes: the second child to arrive at a node
  // merges the node's two child records (boxes, and body tags in their w) and writes the result
  // into the node's slot in its parent.  The parent and the side of the slot depend only on
  // the tree, so they are loaded before the arrival: each level costs the arrival and the
  // children's records, two round trips.
  int node = __ldg(parent + i);
  if (node < n || node >= 2 * n - 1) return;  // malformed parent link
  int pn = node != n ? __ldg(parent + node) : n;
  int side = node != n ? (__ldg(left + pn) == node ? 0 : 1) : 0;
  for (int depth = 0; depth < n; ++depth) {  // a valid tree is at most n - 1 deep
    // the next level's parent and side, loaded while the arrival is in flight (wasted when this
    // thread arrives first)
    const int next = pn;
    const bool next_ok = next != n && next >= n && next < 2 * n - 1;
    const int npn = next_ok ? __ldg(parent + next) : n;
    if (ar_lbvh::arrive(counters + (node - n)) == 0) return;
    const float4* c = nodes[node - n].c;
    const float4 a0 = __ldcg(c), a1 = __ldcg(c + 1), b0 = __ldcg(c + 2), b1 = __ldcg(c + 3);
    if (node == n) return;  // the root's box is not stored anywhere
    if (next != n && !next_ok) return;  // malformed parent link
    const int nside = next_ok && npn >= n && npn < 2 * n - 1 && __ldg(left + npn) != next ? 1 : 0;
    const ar_lbvh::Box6 m = ar_lbvh::merge_boxes(ar_lbvh::Box6{a0.x, a0.y, a0.z, a0.w, a1.x, a1.y},
                                                 ar_lbvh::Box6{b0.x, b0.y, b0.z, b0.w, b1.x, b1.y});
    // both children have arrived, so their tags (the records' last words) are visible like
    // their boxes
    const int tl = __float_as_int(a1.w), tr = __float_as_int(b1.w);
    put_child(nodes, pn - n, side, make_float4(m.lx, m.ly, m.lz, m.hx), make_float2(m.hy, m.hz),
              node, tl == tr ? tl : -1);
    node = next;
    pn = npn;
    side = nside;
  }
}

// Leaves in sorted order: position (w = global body id) and velocity recomputed from the body
// state; the leaf box (position +/- r) goes into its parent's slot, and the thread climbs from
// there (the refit); leaf flags and ranges.
template <bool kOne>
__global__ void __launch_bounds__(256) bvh_leaves_kernel(
    const __grid_constant__ SceneDev one, const SceneDev* __restrict__ table, const int* __restrict__ pscene, int ns, int nt,
    const uint32_t* __restrict__ svals, const int32_t* __restrict__ left,
    const int32_t* __restrict__ parent, float4* __restrict__ spos, float4* __restrict__ svel,
    WideNode* __restrict__ nodes, uint8_t* __restrict__ is_leaf, int32_t* __restrict__ min_r,
    int32_t* __restrict__ max_r, int* __restrict__ counters, const uint32_t* __restrict__ skeys32,
    uint32_t* __restrict__ prev_keys, uint32_t* __restrict__ prev_vals) {
  ar::pdl_wait();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nt; k += gridDim.x * blockDim.x) {
    const int g = (int)__ldg(svals + k);
    if (prev_keys) {  // 32-bit keys: the order the next step's re-sort starts from
      prev_keys[k] = __ldg(skeys32 + k);
      prev_vals[k] = (uint32_t)g;
    }
    const int sc = kOne ? 0 : __ldg(pscene + g);
    const SceneDev& S = scene_at<kOne>(one, table, sc);
    const float4 r4 = __ldg(S.rel + (g - S.poff));
    const int b = __float_as_int(r4.w);
    float3 r, p, v;
    ar_pipe::repose(__ldg(S.quat + b), __ldg(S.pos + b), __ldg(S.vel + b), __ldg(S.ang + b),
                    ar::mk3(r4.x, r4.y, r4.z), &r, &p, &v);
    spos[k] = make_float4(p.x, p.y, p.z, __int_as_float(S.boff + b));
    svel[k] = make_float4(v.x, v.y, v.z, __int_as_float(sc));  // w = scene index
    if (nt >= 2) {
      const float rr = S.r;
      const int pn = __ldg(parent + k);
      put_child(nodes, pn - nt, __ldg(left + pn) == k ? 0 : 1,
                make_float4(p.x - rr, p.y - rr, p.z - rr, p.x + rr), make_float2(p.y + rr, p.z + rr),
                k, S.boff + b);
      refit_from_leaf(k, nt, left, parent, nodes, counters);  // the climb starts right here
    }
    is_leaf[k] = 1;
    min_r[k] = k;
    max_r[k] = k;
  }
}

// Each scene's subtree root.  The scene's leaves [lo, hi] are one subtree, whose root covers
// exactly [lo, hi]; a Karras internal node i has i as one end of its range, so the root is
// internal node lo or internal node hi.  (The walk up from the first leaf is kept only as a
// guard against a malformed tree.)
__global__ void bvh_roots_kernel(const int* __restrict__ poff, int ns, int nt,
                                 const int32_t* __restrict__ parent,
                                 const int32_t* __restrict__ min_r,
                                 const int32_t* __restrict__ max_r, int32_t* __restrict__ roots) {
  ar::pdl_wait();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  const int lo = poff[s], hi = poff[s + 1] - 1;
  if (hi <= lo) {  // zero or one particle: no internal node
    roots[s] = -1;
    return;
  }
  for (const int cand : {nt + lo, nt + hi}) {
    if (cand <= 2 * nt - 2 && min_r[cand] == lo && max_r[cand] == hi) {
      roots[s] = cand;
      return;
    }
  }
  int node = parent[lo];
  for (int depth = 0; depth < nt && node >= 0; ++depth) {
    if (min_r[node] <= lo && max_r[node] >= hi) break;
    node = parent[node];
  }
  roots[s] = node;
}

// DEM gather through the scene's subtree in the reference's visit order
// (collideBVHSoARigidBody, Kernels/RB_BVHKernels.cu:145-214): at a node the overlapping leaf
// children are handled left then right, then the walk goes into the left internal child if it
// overlaps, deferring the right one on a short stack.  Contacts are summed in visit order,
// then the walls.  A scene subtree is at most 30 + 32 levels deep (code bits + index bits),
// so the stack never holds more than 62 entries.
constexpr int kBvhStack = 64;

template <bool kOne>
__global__ void __launch_bounds__(256) bvh_collide_kernel(
    const __grid_constant__ SceneDev one, const SceneDev* __restrict__ table, const int* __restrict__ poff, int ns, int nt,
    const uint32_t* __restrict__ svals, const float4* __restrict__ spos,
    const float4* __restrict__ svel, const WideNode* __restrict__ nodes,
    const int32_t* __restrict__ roots, float4* __restrict__ pforce, int* __restrict__ err) {
  ar::pdl_wait();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nt) return;
  const float4 p4 = __ldg(spos + k);
  const float4 v4 = __ldg(svel + k);
  const int s = kOne ? 0 : __float_as_int(v4.w);
  const SceneDev& S = scene_at<kOne>(one, table, s);
  const float3 pos = ar::xyz(p4), vel = ar::xyz(v4);
  const int body = __float_as_int(p4.w);
  const float rr = S.r;
  const float thr = 2.0f * rr;
  const float thr2_up = nextafterf(thr * thr, INFINITY);
  const float kk = S.k, dmp = S.damping, shr = S.shear, att = S.attraction;
  float3 lin = ar::mk3(0.f, 0.f, 0.f);
  const int root = __ldg(roots + s);
  if (root >= nt) {  // an internal node
    const ar_lbvh::Box q{pos.x - rr, pos.y - rr, pos.z - rr, pos.x + rr, pos.y + rr, pos.z + rr};
    auto visit = [&](int c) {
      const float4 q4 = __ldg(spos + c);
      if (__float_as_int(q4.w) == body) return;
      const float3 rp = ar::sub(ar::xyz(q4), pos);
      const float d2 = ar::dot(rp, rp);
      if (!(d2 < thr2_up)) return;
      const float dist = sqrtf(d2);
      if (!(dist < thr)) return;
      const float3 v2 = ar::xyz(__ldg(svel + c));
      lin = ar::add(lin, ar_dem::spring_force(rp, dist, ar::sub(v2, vel), thr, kk, dmp, shr, att));
    };
    int stack[kBvhStack];
    int top = 0;
    int node = root;
    for (int guard = 2 * nt; guard > 0; --guard) {
      const float4* c = nodes[node - nt].c;
      const float4 a0 = __ldg(c), a1 = __ldg(c + 1), b0 = __ldg(c + 2), b1 = __ldg(c + 3);
      const int lc = __float_as_int(a1.z), rc = __float_as_int(b1.z);
      // a child holding only this particle's body (this particle's own leaf included) is skipped
      const bool ol = __float_as_int(a1.w) != body &&
                      ar_lbvh::overlap(q, ar_lbvh::Box{a0.x, a0.y, a0.z, a0.w, a1.x, a1.y});
      const bool orr = __float_as_int(b1.w) != body &&
                       ar_lbvh::overlap(q, ar_lbvh::Box{b0.x, b0.y, b0.z, b0.w, b1.x, b1.y});
      const bool ll = lc < nt, rl = rc < nt;
      if (ol && ll) visit(lc);
      if (orr && rl) visit(rc);
      const bool tl = ol && !ll, tr = orr && !rl;
      if (!tl && !tr) {
        if (top == 0) break;
        node = stack[--top];
      } else {
        node = tl ? lc : rc;
        if (tl && tr) {
          if (top < kBvhStack) stack[top++] = rc;
          else ar::raise_error(err, ar::kErrOverflow);
        }
      }
    }
  }
  lin = ar::add(lin, ar_pipe::wall_force(S, pos, vel));
  pforce[__ldg(svals + k)] = make_float4(lin.x, lin.y, lin.z, 0.f);
}

// ---- K5: fixed-order body sums, then integration ------------------------------------------
// One warp per body: fixed-order lane sums of F and r x F over the body's particles, xor-tree
// across lanes, totals stored per body.  Then one thread per body integrates (a separate
// kernel, so that the integration runs on every lane instead of lane 0 of each warp).  A scene
// whose step budget is spent (batch step number > end_step) is frozen: its state and sums are
// left untouched.
template <bool kOne>
__global__ void __launch_bounds__(256) body_step_kernel(
    const __grid_constant__ SceneDev one, const SceneDev* __restrict__ table,
    const int* __restrict__ bscene, int bt,
    const float4* __restrict__ pforce, const long long* __restrict__ d_step,
    int* __restrict__ err) {
  ar::pdl_wait();
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const int lane = ar::lane_id();
  const long long step = *d_step;
  for (int gb = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; gb < bt; gb += warps) {
    const SceneDev& S = scene_at<kOne>(one, table, kOne ? 0 : __ldg(bscene + gb));
    if (step > S.end_step) continue;
    const int b = gb - S.boff;
    const int s0 = __ldg(S.offsets + b), s1 = __ldg(S.offsets + b + 1);
    const float4 q = S.quat[b];
    float fx = 0.f, fy = 0.f, fz = 0.f, tx = 0.f, ty = 0.f, tz = 0.f;
    auto add = [&](const float4& f4, const float4& r4) {
      const float3 f = ar::xyz(f4);
      const float3 t = ar::cross(ar::quat_rotate(q, ar::mk3(r4.x, r4.y, r4.z)), f);
      fx += f.x; fy += f.y; fz += f.z;
      tx += t.x; ty += t.y; tz += t.z;
    };
    // two of a lane's particles in flight together, added in the lane's order
    int i = s0 + lane;
    for (; i + 32 < s1; i += 64) {
      const float4 f4a = __ldcs(pforce + S.poff + i), f4b = __ldcs(pforce + S.poff + i + 32);
      const float4 r4a = __ldg(S.rel + i), r4b = __ldg(S.rel + i + 32);
      add(f4a, r4a);
      add(f4b, r4b);
    }
    if (i < s1) add(__ldcs(pforce + S.poff + i), __ldg(S.rel + i));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      fx += __shfl_xor_sync(0xffffffffu, fx, o);
      fy += __shfl_xor_sync(0xffffffffu, fy, o);
      fz += __shfl_xor_sync(0xffffffffu, fz, o);
      tx += __shfl_xor_sync(0xffffffffu, tx, o);
      ty += __shfl_xor_sync(0xffffffffu, ty, o);
      tz += __shfl_xor_sync(0xffffffffu, tz, o);
    }
    if (lane == 0) {
      S.bforce[b] = make_float4(fx, fy, fz, 0.f);
      S.btorque[b] = make_float4(tx, ty, tz, 0.f);
    }
  }
}

template <bool kOne>
__global__ void __launch_bounds__(256) integrate_kernel(
    const __grid_constant__ SceneDev one, const SceneDev* __restrict__ table,
    const int* __restrict__ bscene, int bt,
    const long long* __restrict__ d_step, int* __restrict__ err) {
  ar::pdl_wait();
  const long long step = *d_step;
  for (int gb = blockIdx.x * blockDim.x + threadIdx.x; gb < bt; gb += gridDim.x * blockDim.x) {
    const SceneDev& S = scene_at<kOne>(one, table, kOne ? 0 : __ldg(bscene + gb));
    if (step > S.end_step) continue;
    const int b = gb - S.boff;
    float ib[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) ib[k] = __ldg(S.inv_inertia + 9 * b + k);
    float4 pos = S.pos[b], quat = S.quat[b], vel = S.vel[b], ang = S.ang[b];
    const float4 F4 = S.bforce[b], T4 = S.btorque[b];
    if (!ar_pipe::integrate_body(S, ar::xyz(F4), ar::xyz(T4), __ldg(S.mass + b), ib, &pos, &quat,
                                 &vel, &ang))
      ar::raise_error(err, ar::kErrNaN);
    S.pos[b] = pos;
    S.quat[b] = quat;
    S.vel[b] = vel;
    S.ang[b] = ang;
  }
}

// ---- render hand-off: per-body model matrices -------------------------------------------------
// The matrix GPUintegratorKernel writes for the renderer (Kernels/rigidBodyKernels.cu:322-331):
// glm::mat4 (column-major) holding mat3_cast of the orientation and the centre as translation.
__global__ void __launch_bounds__(256) model_matrices_kernel(const SceneDev* __restrict__ table,
                                                             const int* __restrict__ bscene,
                                                             int bt, float* __restrict__ out) {
  for (int gb = blockIdx.x * blockDim.x + threadIdx.x; gb < bt; gb += gridDim.x * blockDim.x) {
    const SceneDev& S = table[__ldg(bscene + gb)];
    const int b = gb - S.boff;
    const float4 q = S.quat[b], c = S.pos[b];
    float m[9];
    ar_glm::mat3_cast(q, m);
    float4* o = reinterpret_cast<float4*>(out + 16 * (size_t)gb);
    o[0] = make_float4(m[0], m[1], m[2], 0.f);
    o[1] = make_float4(m[3], m[4], m[5], 0.f);
    o[2] = make_float4(m[6], m[7], m[8], 0.f);
    o[3] = make_float4(c.x, c.y, c.z, 1.f);
  }
}

int ceil_log2(uint64_t v) {
  int b = 0;
  while ((1ull << b) < v) ++b;
  return b;
}

}  // namespace

// --------------------------------------------------------------------------------------------
struct ar_scene {
  ar_ctx* ctx = nullptr;
  ar_scene_desc desc{};
  int n = 0, nb = 0;
  float4 *pos = nullptr, *quat = nullptr, *vel = nullptr, *ang = nullptr;
  float4 *bforce = nullptr, *btorque = nullptr, *rel = nullptr;
  float *mass = nullptr, *inv_inertia = nullptr;
  int32_t* offsets = nullptr;
  void* block = nullptr;  // one stream-ordered allocation holding all of the above
  float origin[3], cell[3];
  uint32_t gdim[3];
  ar_batch* solo = nullptr;
  // static point cloud (ar_scene_set_static_cloud): sorted points, normals, cell table
  int cloud_n = 0;
  float4 *cloud_pos = nullptr, *cloud_norm = nullptr;
  uint2* cloud_cells = nullptr;
  // bumped by every change that the batches' scene tables hold (the cloud), so that a batch
  // holding the scene rebuilds its table before its next step
  uint64_t version = 0;
};

struct ar_batch {
  ar_ctx* ctx = nullptr;
  std::vector<ar_scene*> scenes;
  bool table_dirty = true;
  std::vector<uint64_t> seen_version;  // scenes' versions when the table was built
  bool has_cloud = false;              // some scene has a static point cloud
  // capacities
  long cap_n = 0, cap_b = 0, cap_s = 0;
  uint64_t cap_cells = 0;
  size_t cap_sort = 0;
  // buffers
  uint32_t *keys = nullptr, *skeys = nullptr, *svals = nullptr;
  float4 *spos = nullptr, *svel = nullptr, *pforce = nullptr;
  uint2* cells = nullptr;  // {first slot, count | epoch | body tag} per cell
  char* sort_ws = nullptr;
  // re-sort from the previous step's order (grid broad phase): that order, and the workspace
  uint32_t *pkeys = nullptr, *pvals = nullptr;
  uint32_t *rs_head = nullptr, *rs_bstart = nullptr;
  uint2 *rs_movers = nullptr, *rs_grouped = nullptr;
  uint4* rs_thead = nullptr;
  bool order_valid = false;  // pkeys / pvals hold the last step's order of this particle set
  SceneDev* d_table = nullptr;
  SceneDev one{};  // the scene of a one-scene batch (passed to the kernels as a parameter)
  int *d_poff = nullptr, *d_boff = nullptr;
  int *d_pscene = nullptr, *d_bscene = nullptr;  // scene index per particle / body
  long long* d_step = nullptr;   // number of the step being run (incremented by its first kernel)
  long long host_step = 0;       // steps enqueued so far
  std::vector<long long> end_steps;  // per scene: last step that integrates it (empty: none)
  // pinned staging of the scene table, two alternating buffers
  char* h_stage[2] = {nullptr, nullptr};
  size_t h_stage_cap[2] = {0, 0};
  cudaEvent_t stage_ev[2] = {nullptr, nullptr};
  int stage_i = 0;
  // layout
  long nt = 0, bt = 0;
  uint64_t total_cells = 0;
  int key_bits = 1;
  ar_sort::Plan plan{};  // digit passes of the cell-key sort
  // BVH broad phase (allocated only for BVH batches)
  int broadphase = AR_BROADPHASE_GRID;
  long cap_bvh = 0;
  size_t cap_sort64 = 0;
  uint64_t *keys64 = nullptr, *skeys64 = nullptr;
  uint8_t* is_leaf = nullptr;
  int32_t *left = nullptr, *right = nullptr, *parent = nullptr, *min_r = nullptr,
          *max_r = nullptr, *roots = nullptr;
  WideNode* nodes = nullptr;
  int* counters = nullptr;
  char* sort64_ws = nullptr;
  int bvh_key_bits = kMortonBits;
  // graph
  cudaGraphExec_t graph = nullptr;   // one step
  cudaGraphExec_t graph_k = nullptr; // kGraphSteps steps in one graph
  cudaStream_t cap_stream = nullptr;
};

namespace {

void free_batch_buffers(ar_batch* B) {
  cudaFree(B->keys); cudaFree(B->skeys); cudaFree(B->svals);
  cudaFree(B->spos); cudaFree(B->svel); cudaFree(B->pforce);
  cudaFree(B->cells); cudaFree(B->sort_ws);
  cudaFree(B->pkeys); cudaFree(B->pvals); cudaFree(B->rs_head);
  cudaFree(B->rs_bstart); cudaFree(B->rs_movers); cudaFree(B->rs_grouped); cudaFree(B->rs_thead);
  B->pkeys = B->pvals = B->rs_head = B->rs_bstart = nullptr;
  B->rs_movers = B->rs_grouped = nullptr;
  B->rs_thead = nullptr;
  B->order_valid = false;
  cudaFree(B->d_table); cudaFree(B->d_poff); cudaFree(B->d_boff);
  cudaFree(B->d_pscene); cudaFree(B->d_bscene);
  B->d_pscene = B->d_bscene = nullptr;
  B->keys = B->skeys = B->svals = nullptr;
  B->spos = B->svel = B->pforce = nullptr;
  B->cells = nullptr; B->sort_ws = nullptr; B->d_table = nullptr;
  B->d_poff = B->d_boff = nullptr;
  B->cap_n = B->cap_b = B->cap_s = 0;
  B->cap_cells = 0;
  B->cap_sort = 0;
  cudaFree(B->keys64); cudaFree(B->skeys64); cudaFree(B->is_leaf); cudaFree(B->left);
  cudaFree(B->right); cudaFree(B->parent); cudaFree(B->min_r); cudaFree(B->max_r);
  cudaFree(B->roots); cudaFree(B->nodes); cudaFree(B->counters); cudaFree(B->sort64_ws);
  B->keys64 = B->skeys64 = nullptr;
  B->is_leaf = nullptr;
  B->left = B->right = B->parent = B->min_r = B->max_r = B->roots = nullptr;
  B->nodes = nullptr;
  B->counters = nullptr;
  B->sort64_ws = nullptr;
  B->cap_bvh = 0;
  B->cap_sort64 = 0;
}

void drop_graph(ar_batch* B) {
  if (B->graph) cudaGraphExecDestroy(B->graph);
  if (B->graph_k) cudaGraphExecDestroy(B->graph_k);
  B->graph = nullptr;
  B->graph_k = nullptr;
}

template <class T>
bool alloc(T** p, size_t count) {
  if (arh::dev_malloc((void**)p, count * sizeof(T) + 16) != cudaSuccess) {
    cudaGetLastError();
    *p = nullptr;
    return false;
  }
  return true;
}

uint64_t scene_cells(const ar_scene* s) {
  return (uint64_t)s->gdim[0] * s->gdim[1] * s->gdim[2];
}

// Grid of a scene as the kernels see it (cell_base 0).
void scene_dev_grid(const ar_scene* s, SceneDev* d) {
  for (int a = 0; a < 3; ++a) {
    d->origin[a] = s->origin[a];
    d->cell[a] = s->cell[a];
    d->inv_cell[a] = 1.0f / s->cell[a];
  }
  d->cell_pow2 = 1;
  for (int a = 0; a < 3; ++a) {
    int e = 0;
    if (!(std::frexp(s->cell[a], &e) == 0.5f) || !std::isnormal(s->cell[a]) ||
        !std::isnormal(d->inv_cell[a]))
      d->cell_pow2 = 0;
  }
  d->gx = s->gdim[0]; d->gy = s->gdim[1]; d->gz = s->gdim[2];
  d->lx = (uint32_t)ceil_log2(d->gx);
  d->ly = (uint32_t)ceil_log2(d->gy);
  d->cell_base = 0;
}

// (Re)build the scene table and make sure every buffer is large enough.
ar_status prepare(ar_batch* B, cudaStream_t st) {
  if (!B->table_dirty) {
    bool same = B->seen_version.size() == B->scenes.size();
    for (size_t i = 0; same && i < B->scenes.size(); ++i)
      same = B->scenes[i]->version == B->seen_version[i];
    if (same) return AR_OK;
    B->table_dirty = true;
  }
  drop_graph(B);
  B->order_valid = false;  // the particle set may differ: the next step sorts from scratch
  long nt = 0, bt = 0;
  uint64_t cells = 0;
  std::vector<SceneDev> tab;
  std::vector<int> poff, boff;
  B->seen_version.clear();
  B->has_cloud = false;
  for (ar_scene* s : B->scenes) {
    SceneDev d{};
    const ar_scene_desc& D = s->desc;
    for (int a = 0; a < 3; ++a) {
      d.bmin[a] = D.box_min[a];
      d.bmax[a] = D.box_max[a];
      d.g[a] = D.gravity[a];
    }
    scene_dev_grid(s, &d);
    d.r = D.radius; d.dt = D.dt; d.k = D.spring; d.damping = D.damping; d.shear = D.shear;
    d.attraction = D.attraction;
    d.cell_base = (uint32_t)cells;
    d.poff = (int)nt; d.boff = (int)bt; d.n = s->n; d.nb = s->nb;
    d.pos = s->pos; d.quat = s->quat; d.vel = s->vel; d.ang = s->ang;
    d.mass = s->mass; d.inv_inertia = s->inv_inertia; d.offsets = s->offsets; d.rel = s->rel;
    d.bforce = s->bforce; d.btorque = s->btorque;
    d.end_step = B->end_steps.empty() ? LLONG_MAX : B->end_steps[tab.size()];
    if (s->cloud_n > 0) {
      d.cloud_cells = s->cloud_cells;
      d.cloud_pos = s->cloud_pos;
      d.cloud_norm = s->cloud_norm;
      B->has_cloud = true;
    }
    B->seen_version.push_back(s->version);
    tab.push_back(d);
    poff.push_back((int)nt);
    boff.push_back((int)bt);
    nt += s->n;
    bt += s->nb;
    if (D.broadphase == AR_BROADPHASE_GRID) cells += scene_cells(s);
  }
  poff.push_back((int)nt);
  boff.push_back((int)bt);
  if (cells >= (1ull << 32) || nt >= (1l << 30)) {
    arh::set_error("batch too large: %llu cells, %ld particles", (unsigned long long)cells, nt);
    return AR_ERR_INVALID_ARG;
  }
  const int key_bits = std::max(1, ceil_log2(cells));
  const int passes = ar_sort::make_plan(0, key_bits).passes;
  const size_t sort_bytes = ar_sort::layout(std::max(nt, 1l), 4, passes).total;
  const long ns = (long)B->scenes.size();
  bool realloc_needed = nt > B->cap_n || bt > B->cap_b || ns + 1 > B->cap_s ||
                        cells > B->cap_cells || sort_bytes > B->cap_sort;
  if (realloc_needed) {
    cudaStreamSynchronize(st);
    free_batch_buffers(B);
    // growth with head room, so that a batch whose membership changes every tick (a server)
    // rarely reallocates
    long cn = std::max(nt, 1l) + std::max(nt, 1l) / 2, cb = std::max(bt, 1l) + bt / 2 + 8,
         cs = ns + ns / 2 + 8;
    uint64_t cc = std::min<uint64_t>(std::max<uint64_t>(cells, 1) + cells / 4, 1ull << 32);
    size_t csort = ar_sort::layout(cn, 4, passes).total;
    bool ok = alloc(&B->keys, cn) && alloc(&B->skeys, cn) && alloc(&B->svals, cn) &&
              alloc(&B->spos, cn) && alloc(&B->svel, cn) && alloc(&B->pforce, cn) &&
              alloc(&B->cells, cc) && alloc(&B->sort_ws, csort) && alloc(&B->d_table, cs) &&
              alloc(&B->d_poff, cs + 1) && alloc(&B->d_boff, cs + 1) &&
              alloc(&B->d_pscene, cn) && alloc(&B->d_bscene, cb) && alloc(&B->pkeys, cn) &&
              alloc(&B->pvals, cn) &&
              alloc(&B->rs_head, ar_resort::region_words(cn)) &&
              alloc(&B->rs_thead, 2 * ar_resort::tiles_for(cn) + 2) &&
              alloc(&B->rs_bstart, (1 << ar_resort::kBucketLog2) + 1) &&
              alloc(&B->rs_movers, cn) && alloc(&B->rs_grouped, cn);
    if (!ok) {
      free_batch_buffers(B);
      arh::set_error("batch workspace allocation failed (%ld particles, %llu cells)", nt,
                     (unsigned long long)cells);
      return AR_ERR_OOM;
    }
    B->cap_n = cn; B->cap_b = cb; B->cap_s = cs; B->cap_cells = cc; B->cap_sort = csort;
    cudaMemsetAsync(B->cells, 0, cc * sizeof(uint2), st);  // epoch 0: empty
  }
  B->broadphase = ns > 0 ? B->scenes[0]->desc.broadphase : AR_BROADPHASE_GRID;
  if (B->broadphase == AR_BROADPHASE_BVH) {
    B->bvh_key_bits = kMortonBits + std::max(0, ceil_log2((uint64_t)std::max(ns, 1l)));
    const int passes64 = ar_sort::make_plan(0, B->bvh_key_bits).passes;
    const size_t s64 = ar_sort::layout(std::max(nt, 1l), 8, passes64).total;
    if (nt > B->cap_bvh || s64 > B->cap_sort64) {
      cudaStreamSynchronize(st);
      const long cn = B->cap_n;
      const size_t m = 2 * (size_t)cn;
      const size_t csort = ar_sort::layout(cn, 8, passes64).total;
      cudaFree(B->keys64); cudaFree(B->skeys64); cudaFree(B->is_leaf); cudaFree(B->left);
      cudaFree(B->right); cudaFree(B->parent); cudaFree(B->min_r); cudaFree(B->max_r);
      cudaFree(B->roots); cudaFree(B->nodes); cudaFree(B->counters); cudaFree(B->sort64_ws);
      bool ok = alloc(&B->keys64, cn) && alloc(&B->skeys64, cn) && alloc(&B->is_leaf, m) &&
                alloc(&B->left, m) && alloc(&B->right, m) && alloc(&B->parent, m) &&
                alloc(&B->min_r, m) && alloc(&B->max_r, m) && alloc(&B->roots, B->cap_s) &&
                alloc(&B->nodes, cn) && alloc(&B->counters, cn) &&
                alloc(&B->sort64_ws, csort);
      if (!ok) {
        free_batch_buffers(B);
        arh::set_error("BVH workspace allocation failed (%ld particles)", nt);
        return AR_ERR_OOM;
      }
      B->cap_bvh = cn;
      B->cap_sort64 = csort;
    }
  }
  if (ns > 0) {
    // table and offsets -> pinned staging -> device, ordered on the stream without a host
    // wait for the steps in flight (they read the previous table; the copy lands after them).
    // Two staging buffers alternate; a buffer is reused once its previous copy has run.
    const size_t tab_b = tab.size() * sizeof(SceneDev), off_b = poff.size() * sizeof(int);
    const size_t need = tab_b + 2 * off_b;
    const int i = B->stage_i;
    if (B->stage_ev[i]) cudaEventSynchronize(B->stage_ev[i]);
    else cudaEventCreateWithFlags(&B->stage_ev[i], cudaEventDisableTiming);
    if (need > B->h_stage_cap[i]) {
      if (B->h_stage[i]) cudaFreeHost(B->h_stage[i]);
      B->h_stage[i] = nullptr;
      B->h_stage_cap[i] = 0;
      if (arh::host_malloc((void**)&B->h_stage[i], 2 * need) != cudaSuccess) {
        cudaGetLastError();
        arh::set_error("batch prepare: pinned staging allocation failed");
        return AR_ERR_OOM;
      }
      B->h_stage_cap[i] = 2 * need;
    }
    char* h = B->h_stage[i];
    std::memcpy(h, tab.data(), tab_b);
    std::memcpy(h + tab_b, poff.data(), off_b);
    std::memcpy(h + tab_b + off_b, boff.data(), off_b);
    cudaMemcpyAsync(B->d_table, h, tab_b, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(B->d_poff, h + tab_b, off_b, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(B->d_boff, h + tab_b + off_b, off_b, cudaMemcpyHostToDevice, st);
    cudaEventRecord(B->stage_ev[i], st);
    B->stage_i ^= 1;
    const long m = std::max(nt, bt);
    scene_ids_kernel<<<std::min(arh::grid_for(m, 256), 4096u), 256, 0, st>>>(
        B->d_poff, B->d_boff, (int)ns, (int)nt, (int)bt, B->d_pscene, B->d_bscene);
  }
  {
    // the re-sort's tile kernels keep their tiles in shared memory: ask for the full carveout
    // so that eight blocks fit on an SM
    static bool carveout_set = false;
    if (!carveout_set) {
      cudaFuncSetAttribute(ar_resort::place_kernel,
          cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
      cudaGetLastError();
      carveout_set = true;
    }
  }
  B->one = tab.empty() ? SceneDev{} : tab[0];
  B->nt = nt;
  B->bt = bt;
  B->total_cells = cells;
  B->key_bits = key_bits;
  B->plan = ar_sort::make_plan(0, key_bits);
  B->table_dirty = false;
  return arh::check_launch("batch prepare");
}

// The re-sort's workspace for keys of key_bits bits (buckets = the key's top bits).
ar_resort::Work resort_work(ar_batch* B, int key_bits) {
  ar_resort::Work rw{};
  rw.head = B->rs_head;
  rw.tcount = B->rs_head + ar_resort::tcount_offset();
  rw.bits = B->rs_head + ar_resort::bits_offset(B->cap_n);
  rw.thead = B->rs_thead;
  rw.bstart = B->rs_bstart;
  rw.local = B->rs_movers;   // the tiles' movers are dead once grouped by bucket,
  rw.movers = B->rs_movers;  // before the sorted movers are written
  rw.grouped = B->rs_grouped;
  const int nb_log2 = std::min(ar_resort::kBucketLog2, key_bits);
  rw.nb = 1 << nb_log2;
  rw.bshift = key_bits - nb_log2;
  return rw;
}

// The four re-sort kernels: B->keys (this step's keys in particle order) from the previous
// order (pkeys, pvals) into skeys / svals.
void launch_resort(ar_ctx* ctx, ar_batch* B, const ar_resort::Work& rw, cudaStream_t st) {
  const int nt = (int)B->nt;
  const unsigned tiles = (unsigned)ar_resort::tiles_for(nt);
  const unsigned wpb = ar_resort::kWarps;  // warps per block: one per tile / bucket
  arh::launch_pdl(ar_resort::leavers_kernel, dim3(tiles), dim3(ar_resort::kThreads), 0, st,
      (const uint32_t*)B->pkeys, (const uint32_t*)B->pvals, (const uint32_t*)B->keys, nt, rw);
  arh::launch_pdl(ar_resort::bucket_kernel, dim3((tiles + wpb - 1) / wpb),
      dim3(ar_resort::kThreads), 0, st, (const uint32_t*)B->pkeys, (const uint32_t*)B->pvals,
      nt, (int)tiles, rw);
  arh::launch_pdl(ar_resort::bucket_sort_kernel, dim3((rw.nb + wpb - 1) / wpb),
      dim3(ar_resort::kThreads), 0, st, rw);
  arh::launch_pdl(ar_resort::place_kernel, dim3(tiles), dim3(ar_resort::kThreads), 0, st,
      (const uint32_t*)B->pkeys, (const uint32_t*)B->pvals, nt, rw, B->skeys, B->svals,
      ctx->d_err);
}

// Stage boundaries for ar_step_profile: events[0] before the step, events[i] after stage i.
// Grid: clear (sort histogram head, cell-table slice) | cell keys + histogram | sort |
// scatter + cell table | collide | body sums + integration.  BVH: clear (refit counters) | Morton keys
// | sort | tree (Karras nodes, leaves, scene roots, refit) | collide | body sums + integration.
constexpr int kStages = 6;

ar_status enqueue_step(ar_batch* B, cudaStream_t st, cudaEvent_t* ev = nullptr) {
  if (B->nt == 0) return AR_OK;
  ar_ctx* ctx = B->ctx;
  const int ns = (int)B->scenes.size();
  const int nt = (int)B->nt, bt = (int)B->bt;
  auto mark = [&](int i) {
    if (ev) cudaEventRecord(ev[i], st);
  };
  // collision block size: the BVH walk runs 64-thread blocks (2M pile: 340 -> 336 us against
  // 128), the grid gather 128 (32 to 128 measured within 1 us of one another)
  int bs = B->broadphase == AR_BROADPHASE_BVH ? 64 : 128;
  if (ns > 0 && B->scenes[0]->desc.block_size > 0) bs = B->scenes[0]->desc.block_size;
  const unsigned gp = std::min(arh::grid_for(nt, 256), (unsigned)ctx->num_sms * 8);
  const unsigned g5 = arh::grid_for((long)bt * 32, 256);
  // a batch of one scene launches the kernels that take its descriptor as a parameter
  const bool one = ns == 1;
#define AR_LAUNCH_ONE(kern, grid, block, ...)                                              \
  do {                                                                                      \
    if (one) arh::launch_pdl(kern<true>, grid, block, 0, st, B->one, __VA_ARGS__);          \
    else arh::launch_pdl(kern<false>, grid, block, 0, st, B->one, __VA_ARGS__);            \
  } while (0)
  mark(0);
  if (B->broadphase == AR_BROADPHASE_BVH) {
    cudaMemsetAsync(B->counters, 0, (size_t)nt * sizeof(int), st);  // refit arrival counters
    mark(1);
    // keys of at most 32 bits (up to 4 scenes) are sorted as uint32: half the bytes per pass
    const bool k32 = B->bvh_key_bits <= 32;
    if (k32 && one)
      arh::launch_pdl(morton_key_kernel<uint32_t, true>, dim3(gp), dim3(256), 0, st, B->one,
          B->d_table, B->d_pscene, ns, nt, B->keys, B->d_step);
    else if (k32)
      arh::launch_pdl(morton_key_kernel<uint32_t, false>, dim3(gp), dim3(256), 0, st, B->one,
          B->d_table, B->d_pscene, ns, nt, B->keys, B->d_step);
    else
      arh::launch_pdl(morton_key_kernel<uint64_t, false>, dim3(gp), dim3(256), 0, st, B->one,
          B->d_table, B->d_pscene, ns, nt, B->keys64, B->d_step);
    mark(2);
    // 32-bit keys are re-sorted from the last step's order once there is one (as in the grid
    // step; ar_resort.cuh), 64-bit keys radix-sorted every step
    const bool resort32 = k32 && B->order_valid;
    if (resort32) {
      const ar_resort::Work rw = resort_work(B, B->bvh_key_bits);
      cudaMemsetAsync(rw.head, 0, ar_resort::cleared_words() * 4, st);
      launch_resort(ctx, B, rw, st);
    } else {
      ar_status s = k32 ? ar_sort::sort_u32(ctx, B->keys, nullptr, B->skeys, B->svals, nt, 0,
                                            B->bvh_key_bits, st, B->sort64_ws, B->cap_sort64)
                        : ar_sort::sort_u64(ctx, B->keys64, nullptr, B->skeys64, B->svals, nt, 0,
                                            B->bvh_key_bits, st, B->sort64_ws, B->cap_sort64);
      if (s != AR_OK) return s;
    }
    mark(3);
    const dim3 gb(arh::grid_for(std::max(nt - 1, 1), 256));
    if (k32)
      arh::launch_pdl(bvh_build_kernel<ar_lbvh::Lcp32Scene>, gb, dim3(256), 0, st,
          ar_lbvh::Lcp32Scene{B->skeys, nt, B->d_poff, kMortonBits}, nt, B->is_leaf, B->left,
          B->right, B->parent, B->min_r, B->max_r, B->nodes);
    else
      arh::launch_pdl(bvh_build_kernel<ar_lbvh::Lcp64Scene>, gb, dim3(256), 0, st,
          ar_lbvh::Lcp64Scene{B->skeys64, nt, B->d_poff, kMortonBits}, nt, B->is_leaf, B->left,
          B->right, B->parent, B->min_r, B->max_r, B->nodes);
    // one thread per leaf: each climbs after storing its leaf (128-thread blocks: a block holds
    // its SM slot until its last climber is done; 2M pile tree stage 288 -> 278 us against 256)
    AR_LAUNCH_ONE(bvh_leaves_kernel, dim3(arh::grid_for(nt, 128)), dim3(128), B->d_table,
        B->d_pscene, ns, nt, B->svals, B->left, B->parent, B->spos, B->svel, B->nodes, B->is_leaf,
        B->min_r, B->max_r, B->counters, (const uint32_t*)B->skeys, k32 ? B->pkeys : nullptr,
        k32 ? B->pvals : nullptr);
    arh::launch_pdl(bvh_roots_kernel, dim3(arh::grid_for(ns, 128)), dim3(128), 0, st, B->d_poff, ns,
        nt, B->parent, B->min_r, B->max_r, B->roots);
    mark(4);
    AR_LAUNCH_ONE(bvh_collide_kernel, dim3(arh::grid_for(nt, bs)), dim3(bs), B->d_table,
        B->d_poff, ns, nt, B->svals, B->spos, B->svel, B->nodes, B->roots, B->pforce, ctx->d_err);
    mark(5);
    AR_LAUNCH_ONE(body_step_kernel, dim3(g5), dim3(256), B->d_table, B->d_bscene, bt,
        B->pforce, B->d_step, ctx->d_err);
    AR_LAUNCH_ONE(integrate_kernel, dim3(arh::grid_for(bt, 128)), dim3(128), B->d_table,
        B->d_bscene, bt, B->d_step, ctx->d_err);
    mark(6);
    B->order_valid = k32;  // the leaves kernel left this step's order in pkeys / pvals
    return arh::check_launch("step (BVH)");  // (AR_LAUNCH_ONE is undefined after the grid path)
  }
  // With the last step's order of this particle set at hand, the keys are re-sorted from it
  // (ar_resort); otherwise (first step after a change of the member list) they are radix-sorted
  // from scratch, with the histogram accumulated in K1.
  const bool resort = B->order_valid;
  const ar_resort::Work rw = resort ? resort_work(B, B->key_bits) : ar_resort::Work{};
  const long head16 = resort ? (long)(ar_resort::cleared_words() / 4)
                             : (long)(ar_sort::clear_bytes(nt, B->plan.passes) / 16);
  arh::launch_pdl(step_clear_kernel, dim3(ctx->num_sms * 2), dim3(256), 0, st,
      resort ? (uint4*)B->rs_head : (uint4*)B->sort_ws, head16, B->cells, B->cap_cells, B->d_step);
  mark(1);
  {
    const dim3 gk(std::min(arh::grid_for(nt, kK1Threads), (unsigned)ctx->num_sms * 4));
    auto* k1 = one ? (resort ? grid_keys_kernel<true, false> : grid_keys_kernel<true, true>)
                   : (resort ? grid_keys_kernel<false, false> : grid_keys_kernel<false, true>);
    arh::launch_pdl(k1, gk, dim3(kK1Threads), 0, st, B->one, B->d_table, B->d_pscene, nt, B->keys,
        (uint32_t*)B->sort_ws, B->plan, B->d_step);
  }
  mark(2);
  if (resort) {
    launch_resort(ctx, B, rw, st);
  } else {
    // cell keys in particle order: a warp's keys share few digits, so match.any ranking
    ar_status s = ar_sort::sort_u32(ctx, B->keys, nullptr, B->skeys, B->svals, nt, 0,
                                    B->key_bits, st, B->sort_ws, B->cap_sort, true, true);
    if (s != AR_OK) return s;
  }
  mark(3);
  AR_LAUNCH_ONE(scatter_kernel, dim3(gp), dim3(256), B->d_table, B->d_pscene, nt, B->skeys,
      B->svals, B->cells, B->spos, B->svel, B->pkeys, B->pvals, B->d_step);
  mark(4);
  AR_LAUNCH_ONE(collide_kernel, dim3(arh::grid_for(nt, bs)), dim3(bs), B->d_table, nt,
      B->skeys, B->svals, B->cells, B->spos, B->svel, B->pforce, B->d_step);
  if (B->has_cloud)
    AR_LAUNCH_ONE(cloud_collide_kernel, dim3(arh::grid_for(nt, 128)), dim3(128), B->d_table, nt,
        B->skeys, B->svals, B->spos, B->svel, B->pforce);
  mark(5);
  AR_LAUNCH_ONE(body_step_kernel, dim3(g5), dim3(256), B->d_table, B->d_bscene, bt,
      B->pforce, B->d_step, ctx->d_err);
  AR_LAUNCH_ONE(integrate_kernel, dim3(arh::grid_for(bt, 128)), dim3(128), B->d_table,
      B->d_bscene, bt, B->d_step, ctx->d_err);
  mark(6);
#undef AR_LAUNCH_ONE
  B->order_valid = true;  // the scatter leaves this step's order in pkeys / pvals
  return arh::check_launch("step");
}

// Run n_steps eagerly with events between the stages; average milliseconds per stage.
ar_status profile_steps(ar_batch* B, int n_steps, float* stage_ms, cudaStream_t st) {
  cudaEvent_t ev[kStages + 1];
  for (auto& e : ev) cudaEventCreate(&e);
  double acc[kStages] = {0};
  ar_status s = AR_OK;
  for (int i = 0; i < n_steps && s == AR_OK; ++i) {
    s = enqueue_step(B, st, ev);
    if (s != AR_OK) break;
    ++B->host_step;
    if (cudaEventSynchronize(ev[kStages]) != cudaSuccess) {
      s = arh::check_launch("profile");
      break;
    }
    for (int k = 0; k < kStages; ++k) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
      acc[k] += ms;
    }
  }
  for (auto& e : ev) cudaEventDestroy(e);
  for (int k = 0; k < kStages; ++k) stage_ms[k] = n_steps > 0 ? (float)(acc[k] / n_steps) : 0.f;
  return s;
}

constexpr int kGraphSteps = 8;

// Capture `steps` consecutive steps into *exec (once; kept until the member list changes).
// Capture records without executing; the graph's launches on the stream it is replayed on are
// ordered after the work already queued there (table uploads, clears).
ar_status capture_steps(ar_batch* B, int steps, cudaGraphExec_t* exec) {
  if (*exec) return AR_OK;
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(B->cap_stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    arh::set_error("cudaStreamBeginCapture failed");
    return AR_ERR_CUDA;
  }
  ar_status es = AR_OK;
  for (int i = 0; i < steps && es == AR_OK; ++i) es = enqueue_step(B, B->cap_stream);
  cudaError_t ce = cudaStreamEndCapture(B->cap_stream, &g);
  if (es != AR_OK || ce != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    arh::set_error("step capture failed (%s)", cudaGetErrorString(ce));
    return es != AR_OK ? es : AR_ERR_CUDA;
  }
  ce = cudaGraphInstantiate(exec, g, 0);
  cudaGraphDestroy(g);
  if (ce != cudaSuccess) {
    *exec = nullptr;
    arh::set_error("cudaGraphInstantiate failed (%s)", cudaGetErrorString(ce));
    return AR_ERR_CUDA;
  }
  return AR_OK;
}

ar_status batch_step(ar_ctx* ctx, ar_batch* B, int n_steps, int use_graph, cudaStream_t st) {
  ar_status s = prepare(B, st);
  if (s != AR_OK) return s;
  if (B->nt == 0 || n_steps <= 0) return AR_OK;
  const bool resorts = B->broadphase == AR_BROADPHASE_GRID || B->bvh_key_bits <= 32;
  if (resorts && !B->order_valid) {
    // the first step after a change of the member list sorts from scratch, outside the graphs
    // (which hold re-sorting steps)
    if ((s = enqueue_step(B, st)) != AR_OK) return s;
    ++B->host_step;
    if (--n_steps == 0) return AR_OK;
  }
  if (!use_graph) {
    for (int i = 0; i < n_steps; ++i) {
      if ((s = enqueue_step(B, st)) != AR_OK) return s;
      ++B->host_step;
    }
    return AR_OK;
  }
  if (!B->cap_stream &&
      cudaStreamCreateWithFlags(&B->cap_stream, cudaStreamNonBlocking) != cudaSuccess) {
    arh::set_error("capture stream creation failed");
    return AR_ERR_CUDA;
  }
  // runs of kGraphSteps steps replay one graph holding them all: inside a graph the steps'
  // launches keep their programmatic dependencies, so each step's first kernel overlaps the
  // previous step's last one, which a graph boundary would not allow
  const bool many = n_steps >= kGraphSteps;
  if ((s = capture_steps(B, 1, &B->graph)) != AR_OK) return s;
  if (many && (s = capture_steps(B, kGraphSteps, &B->graph_k)) != AR_OK) return s;
  int left = n_steps;
  for (; many && left >= kGraphSteps; left -= kGraphSteps) {
    if (cudaGraphLaunch(B->graph_k, st) != cudaSuccess) return arh::check_launch("graph launch");
    B->host_step += kGraphSteps;
  }
  for (; left > 0; --left) {
    if (cudaGraphLaunch(B->graph, st) != cudaSuccess) return arh::check_launch("graph launch");
    ++B->host_step;
  }
  return arh::check_launch("graph launch");
}

uint32_t next_pow2(uint64_t v) {
  uint32_t p = 1;
  while (p < v && p < (1u << 31)) p <<= 1;
  return p;
}

// Grid of a scene: cell edge (default 2r), origin at the box minimum, cells per axis the next
// power of two covering the box (or the given log2), then halved on the largest axis while the
// total exceeds max(2^12, next_pow2(8 N)) -- the wrap keeps any size correct.
void scene_grid(const ar_scene_desc& D, float origin[3], float cell[3], uint32_t g[3]) {
  const float c = D.cell_size > 0.f ? D.cell_size : 2.f * D.radius;
  for (int a = 0; a < 3; ++a) {
    origin[a] = D.box_min[a];
    cell[a] = c;
    if (D.grid_log2[a] > 0) {
      g[a] = 1u << D.grid_log2[a];
    } else {
      double ext = (double)D.box_max[a] - (double)D.box_min[a];
      uint64_t cells = (uint64_t)std::ceil(ext / c);
      g[a] = std::max<uint32_t>(4, next_pow2(std::max<uint64_t>(cells, 1)));
    }
  }
  if (D.grid_log2[0] > 0 || D.grid_log2[1] > 0 || D.grid_log2[2] > 0) return;
  const uint64_t cap = std::max<uint64_t>(1ull << 12, next_pow2(8ull * std::max(D.num_particles, 1)));
  while ((uint64_t)g[0] * g[1] * g[2] > cap) {
    int a = 0;
    for (int k = 1; k < 3; ++k) if (g[k] > g[a]) a = k;
    if (g[a] <= 4) break;
    g[a] >>= 1;
  }
}

}  // namespace

extern "C" {

size_t ar_scene_footprint(const ar_scene_desc* d) {
  if (!d) return 0;
  const size_t n = (size_t)std::max(d->num_particles, 0), b = (size_t)std::max(d->num_bodies, 0);
  const size_t per_body = 16 * 6 + 4 + 36 + 4;
  const size_t shared = 16 /*rel*/ + 16 * 3 /*spos svel pforce*/ + 4 /*svals*/ + 1;
  if (d->broadphase == AR_BROADPHASE_BVH) {
    const size_t per_particle = shared + 8 * 2 /*keys64*/ + 12 /*sort tmp*/ +
                                2 * (1 + 4 * 5) /*tree*/ + 2 * 32 /*boxes*/ + 4 /*counters*/;
    return n * per_particle + b * per_body + 4096;
  }
  const size_t per_particle = shared + 4 * 2 /*keys*/ + 8 /*sort tmp*/;
  return n * per_particle + b * per_body + (size_t)ar_scene_cells(d) * sizeof(uint2) + 4096;
}

uint64_t ar_scene_cells(const ar_scene_desc* d) {
  if (!d || d->broadphase != AR_BROADPHASE_GRID) return 0;
  float o[3], c[3];
  uint32_t g[3];
  scene_grid(*d, o, c, g);
  return (uint64_t)g[0] * g[1] * g[2];
}

}  // extern "C"

namespace {
// Bytes of a scene's device block: body centre, orientation, velocity, angular velocity (float4
// each, adjacent, so that the four move in one copy), force and torque sums, mass, inverse
// inertia, body offsets and particle offsets; the groups 256-byte aligned.
size_t scene_block_bytes(int nb, int n, size_t sizes[5]) {
  const size_t a4 = 64 * (size_t)nb, a1 = 16 * (size_t)nb;
  sizes[0] = ((a4 + 255) & ~(size_t)255) + 2 * ((a1 + 255) & ~(size_t)255);
  sizes[1] = 4 * (size_t)nb;
  sizes[2] = 36 * (size_t)nb;
  sizes[3] = 4 * (size_t)(nb + 1);
  sizes[4] = 16 * (size_t)n;
  size_t total = 0;
  for (int i = 0; i < 5; ++i) total += (sizes[i] + 255) & ~(size_t)255;
  return total;
}

// One allocation from the stream-ordered pool for the scene's arrays, carved in the order of
// scene_block_bytes.  False (block left null) when the pool has no room.
bool alloc_scene_block(ar_scene* s, cudaStream_t st) {
  size_t sizes[5];
  const size_t total = scene_block_bytes(s->nb, s->n, sizes);
  if (arh::dev_malloc_async(&s->block, total, st) != cudaSuccess) {
    cudaGetLastError();
    s->block = nullptr;
    return false;
  }
  char* b = (char*)s->block;
  const size_t a1 = 16 * (size_t)s->nb, a4 = (4 * a1 + 255) & ~(size_t)255;
  float4** state[4] = {&s->pos, &s->quat, &s->vel, &s->ang};
  for (int i = 0; i < 4; ++i) *state[i] = (float4*)(b + i * a1);
  s->bforce = (float4*)(b + a4);
  s->btorque = (float4*)(b + a4 + ((a1 + 255) & ~(size_t)255));
  b += (sizes[0] + 255) & ~(size_t)255;
  s->mass = (float*)b;
  b += (sizes[1] + 255) & ~(size_t)255;
  s->inv_inertia = (float*)b;
  b += (sizes[2] + 255) & ~(size_t)255;
  s->offsets = (int32_t*)b;
  b += (sizes[3] + 255) & ~(size_t)255;
  s->rel = (float4*)b;
  return true;
}
}  // namespace

extern "C" {

ar_status ar_scene_create(ar_ctx* ctx, const ar_scene_desc* desc, const ar_scene_init* init,
                          ar_stream_t stream, ar_scene** out) {
  if (!ctx || !desc || !init || !out) return AR_ERR_INVALID_ARG;
  *out = nullptr;
  const ar_scene_desc& D = *desc;
  if (D.num_bodies <= 0 || D.num_particles <= 0 || !(D.radius > 0.f) || !(D.dt > 0.f)) {
    arh::set_error("ar_scene_create: need bodies, particles, radius > 0 and dt > 0");
    return AR_ERR_INVALID_ARG;
  }
  if (D.broadphase != AR_BROADPHASE_GRID && D.broadphase != AR_BROADPHASE_BVH) {
    arh::set_error("ar_scene_create: unknown broadphase %d", D.broadphase);
    return AR_ERR_INVALID_ARG;
  }
  for (int a = 0; a < 3; ++a)
    if (D.grid_log2[a] < 0 || D.grid_log2[a] > 20) return AR_ERR_INVALID_ARG;
  if (D.block_size != 0 && (D.block_size < 32 || D.block_size > 256 || D.block_size % 32)) {
    arh::set_error("ar_scene_create: block_size must be a multiple of 32 in [32, 256]");
    return AR_ERR_INVALID_ARG;
  }
  if (!init->body_pos4 || !init->body_quat4 || !init->body_vel4 || !init->body_angvel4 ||
      !init->body_mass || !init->body_inv_inertia9 || !init->body_offsets || !init->particle_rel4)
    return AR_ERR_INVALID_ARG;
  const int nb = D.num_bodies, n = D.num_particles;
  if (init->body_offsets[0] != 0 || init->body_offsets[nb] != n) {
    arh::set_error("ar_scene_create: body_offsets must run from 0 to num_particles");
    return AR_ERR_INVALID_ARG;
  }
  for (int b = 0; b < nb; ++b)
    if (init->body_offsets[b + 1] < init->body_offsets[b]) {
      arh::set_error("ar_scene_create: body_offsets must be non-decreasing");
      return AR_ERR_INVALID_ARG;
    }
  ar_scene* s = new ar_scene();
  s->ctx = ctx;
  s->desc = D;
  s->n = n;
  s->nb = nb;
  scene_grid(D, s->origin, s->cell, s->gdim);
  cudaStream_t st = arh::stream(stream);
  // one allocation from the stream-ordered pool (no device-wide synchronisation), carved into
  // 256-byte aligned arrays
  if (!alloc_scene_block(s, st)) {
    ar_scene_destroy(s);
    arh::set_error("ar_scene_create: out of device memory");
    return AR_ERR_OOM;
  }
  // particle rel with the body index in w
  std::vector<float4> rel(n);
  for (int b = 0; b < nb; ++b)
    for (int i = init->body_offsets[b]; i < init->body_offsets[b + 1]; ++i) {
      const float* r = init->particle_rel4 + 4 * (size_t)i;
      float w;
      std::memcpy(&w, &b, 4);
      rel[i] = make_float4(r[0], r[1], r[2], w);
    }
  cudaMemcpyAsync(s->pos, init->body_pos4, 16 * (size_t)nb, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s->quat, init->body_quat4, 16 * (size_t)nb, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s->vel, init->body_vel4, 16 * (size_t)nb, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s->ang, init->body_angvel4, 16 * (size_t)nb, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s->mass, init->body_mass, 4 * (size_t)nb, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s->inv_inertia, init->body_inv_inertia9, 36 * (size_t)nb, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s->offsets, init->body_offsets, 4 * (size_t)(nb + 1), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(s->rel, rel.data(), 16 * (size_t)n, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(s->bforce, 0, 16 * (size_t)nb, st);
  cudaMemsetAsync(s->btorque, 0, 16 * (size_t)nb, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    arh::set_error("ar_scene_create: %s", cudaGetErrorString(e));
    ar_scene_destroy(s);
    return AR_ERR_CUDA;
  }
  *out = s;
  return AR_OK;
}

ar_status ar_scene_clone_async(const ar_scene* proto, ar_stream_t stream, ar_scene** out) {
  if (!proto || !out || !proto->block) return AR_ERR_INVALID_ARG;
  *out = nullptr;
  ar_scene* s = new ar_scene();
  s->ctx = proto->ctx;
  s->desc = proto->desc;
  s->n = proto->n;
  s->nb = proto->nb;
  for (int a = 0; a < 3; ++a) {
    s->origin[a] = proto->origin[a];
    s->cell[a] = proto->cell[a];
    s->gdim[a] = proto->gdim[a];
  }
  cudaStream_t st = arh::stream(stream);
  if (!alloc_scene_block(s, st)) {
    ar_scene_destroy(s);
    arh::set_error("ar_scene_clone_async: out of device memory");
    return AR_ERR_OOM;
  }
  size_t sizes[5];
  cudaMemcpyAsync(s->block, proto->block, scene_block_bytes(s->nb, s->n, sizes),
                  cudaMemcpyDeviceToDevice, st);
  *out = s;
  return arh::check_launch("ar_scene_clone_async");
}

static void free_cloud(ar_scene* s) {
  cudaFree(s->cloud_pos);
  cudaFree(s->cloud_norm);
  cudaFree(s->cloud_cells);
  s->cloud_pos = s->cloud_norm = nullptr;
  s->cloud_cells = nullptr;
  s->cloud_n = 0;
}

ar_status ar_scene_destroy(ar_scene* s) {
  if (!s) return AR_ERR_INVALID_ARG;
  if (s->solo) ar_batch_destroy(s->solo);
  if (s->block) cudaFree(s->block);  // waits for the device, like any cudaFree
  free_cloud(s);
  delete s;
  return AR_OK;
}

ar_status ar_scene_destroy_async(ar_scene* s, ar_stream_t stream) {
  if (!s) return AR_ERR_INVALID_ARG;
  if (s->solo) ar_batch_destroy(s->solo);
  if (s->cloud_n > 0) {  // the cloud is freed synchronously (it is not stream-ordered memory)
    cudaStreamSynchronize(arh::stream(stream));
    free_cloud(s);
  }
  if (s->block && cudaFreeAsync(s->block, arh::stream(stream)) != cudaSuccess) {
    delete s;
    return arh::check_launch("ar_scene_destroy_async");
  }
  delete s;
  return AR_OK;
}

ar_status ar_scene_set_static_cloud(ar_ctx* ctx, ar_scene* s, const float* cloud_pos4,
                                    const float* cloud_norm4, int num_points,
                                    ar_stream_t stream) {
  if (!ctx || !s || num_points < 0 || (num_points > 0 && (!cloud_pos4 || !cloud_norm4)))
    return AR_ERR_INVALID_ARG;
  if (s->desc.broadphase != AR_BROADPHASE_GRID) {
    arh::set_error("ar_scene_set_static_cloud: a static cloud needs the grid broad phase");
    return AR_ERR_INVALID_ARG;
  }
  if (num_points > 0 && (((uintptr_t)cloud_pos4 | (uintptr_t)cloud_norm4) & 15u) != 0) {
    arh::set_error("ar_scene_set_static_cloud: pointers must be 16-byte aligned");
    return AR_ERR_INVALID_ARG;
  }
  // steps in flight, on any stream, may still read the old cloud
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    arh::set_error("ar_scene_set_static_cloud: %s", cudaGetErrorString(e));
    return AR_ERR_CUDA;
  }
  free_cloud(s);
  ++s->version;  // every batch holding the scene rebuilds its table (and graphs)
  if (num_points == 0) return AR_OK;
  cudaStream_t st = arh::stream(stream);
  const int m = num_points;
  SceneDev d{};
  scene_dev_grid(s, &d);
  const uint64_t cells = scene_cells(s);
  const int key_bits = std::max(1, ceil_log2(cells));
  const size_t ws_bytes = ar_sort::layout(m, 4, ar_sort::make_plan(0, key_bits).passes).total;
  uint32_t *keys = nullptr, *skeys = nullptr, *sidx = nullptr;
  char* ws = nullptr;
  ar_status r = AR_OK;
  if (!(alloc(&keys, m) && alloc(&skeys, m) && alloc(&sidx, m) && alloc(&ws, ws_bytes) &&
        alloc(&s->cloud_pos, m) && alloc(&s->cloud_norm, m) && alloc(&s->cloud_cells, cells))) {
    arh::set_error("ar_scene_set_static_cloud: out of device memory (%d points, %llu cells)", m,
                   (unsigned long long)cells);
    r = AR_ERR_OOM;
  } else {
    cudaMemsetAsync(s->cloud_cells, 0, cells * sizeof(uint2), st);  // every cell empty
    cloud_keys_kernel<<<arh::grid_for(m, 256), 256, 0, st>>>(d, (const float4*)cloud_pos4, m,
                                                             keys);
    r = ar_sort::sort_u32(ctx, keys, nullptr, skeys, sidx, m, 0, key_bits, st, ws, ws_bytes);
    if (r == AR_OK) {
      cloud_place_kernel<<<arh::grid_for(m, 256), 256, 0, st>>>(
          (const float4*)cloud_pos4, (const float4*)cloud_norm4, skeys, sidx, m, s->cloud_pos,
          s->cloud_norm, s->cloud_cells);
      r = arh::check_launch("ar_scene_set_static_cloud");
    }
    if (r == AR_OK && (e = cudaStreamSynchronize(st)) != cudaSuccess) {
      arh::set_error("ar_scene_set_static_cloud: %s", cudaGetErrorString(e));
      r = AR_ERR_CUDA;
    }
  }
  cudaFree(keys); cudaFree(skeys); cudaFree(sidx); cudaFree(ws);
  if (r != AR_OK) {
    free_cloud(s);
    return r;
  }
  s->cloud_n = m;
  return AR_OK;
}

ar_status ar_scene_download_async(ar_scene* s, float* h_pos4, float* h_quat4, float* h_vel4,
                                  float* h_ang4, ar_stream_t stream) {
  if (!s) return AR_ERR_INVALID_ARG;
  cudaStream_t st = arh::stream(stream);
  const size_t bytes = 16 * (size_t)s->nb;
  if (h_pos4) cudaMemcpyAsync(h_pos4, s->pos, bytes, cudaMemcpyDeviceToHost, st);
  if (h_quat4) cudaMemcpyAsync(h_quat4, s->quat, bytes, cudaMemcpyDeviceToHost, st);
  if (h_vel4) cudaMemcpyAsync(h_vel4, s->vel, bytes, cudaMemcpyDeviceToHost, st);
  if (h_ang4) cudaMemcpyAsync(h_ang4, s->ang, bytes, cudaMemcpyDeviceToHost, st);
  return arh::check_launch("ar_scene_download_async");
}

ar_status ar_scene_download(ar_scene* s, float* h_pos4, float* h_quat4, float* h_vel4,
                            float* h_ang4, ar_stream_t stream) {
  ar_status r = ar_scene_download_async(s, h_pos4, h_quat4, h_vel4, h_ang4, stream);
  if (r != AR_OK) return r;
  cudaError_t e = cudaStreamSynchronize(arh::stream(stream));
  if (e != cudaSuccess) {
    arh::set_error("ar_scene_download: %s", cudaGetErrorString(e));
    return AR_ERR_CUDA;
  }
  return AR_OK;
}

ar_status ar_scene_get_view(ar_scene* s, ar_scene_view* v) {
  if (!s || !v) return AR_ERR_INVALID_ARG;
  v->num_bodies = s->nb;
  v->num_particles = s->n;
  v->body_pos4 = (float*)s->pos; v->body_quat4 = (float*)s->quat;
  v->body_vel4 = (float*)s->vel; v->body_angvel4 = (float*)s->ang;
  v->body_mass = s->mass; v->body_inv_inertia9 = s->inv_inertia; v->body_offsets = s->offsets;
  v->particle_rel4 = (float*)s->rel;
  v->body_force4 = (float*)s->bforce; v->body_torque4 = (float*)s->btorque;
  return AR_OK;
}

ar_status ar_scene_grid_info(ar_scene* s, float origin[3], float cell[3], uint32_t dims[3]) {
  if (!s) return AR_ERR_INVALID_ARG;
  for (int a = 0; a < 3; ++a) {
    if (origin) origin[a] = s->origin[a];
    if (cell) cell[a] = s->cell[a];
    if (dims) dims[a] = s->gdim[a];
  }
  return AR_OK;
}

static ar_status ensure_solo(ar_scene* s) {
  if (s->solo) return AR_OK;
  ar_status st = ar_batch_create(s->ctx, &s->solo);
  if (st != AR_OK) return st;
  return ar_batch_set_scenes(s->solo, &s, 1);
}

ar_status ar_step(ar_ctx* ctx, ar_scene* s, int n_steps, int use_graph, ar_stream_t stream) {
  if (!ctx || !s || n_steps < 0) return AR_ERR_INVALID_ARG;
  ar_status st = ensure_solo(s);
  if (st != AR_OK) return st;
  return batch_step(ctx, s->solo, n_steps, use_graph, arh::stream(stream));
}

ar_status ar_step_profile(ar_ctx* ctx, ar_scene* s, int n_steps, float* h_stage_ms,
                          ar_stream_t stream) {
  if (!ctx || !s || n_steps < 0 || !h_stage_ms) return AR_ERR_INVALID_ARG;
  ar_status st = ensure_solo(s);
  if (st != AR_OK) return st;
  cudaStream_t cs = arh::stream(stream);
  if ((st = prepare(s->solo, cs)) != AR_OK) return st;
  return profile_steps(s->solo, n_steps, h_stage_ms, cs);
}

ar_status ar_batch_profile(ar_ctx* ctx, ar_batch* B, int n_steps, float* h_stage_ms,
                           ar_stream_t stream) {
  if (!ctx || !B || n_steps < 0 || !h_stage_ms) return AR_ERR_INVALID_ARG;
  cudaStream_t cs = arh::stream(stream);
  ar_status st = prepare(B, cs);
  if (st != AR_OK) return st;
  return profile_steps(B, n_steps, h_stage_ms, cs);
}

ar_status ar_scene_upload(ar_scene* s, const float* h_pos4, const float* h_quat4,
                          const float* h_vel4, const float* h_ang4, ar_stream_t stream) {
  if (!s) return AR_ERR_INVALID_ARG;
  cudaStream_t st = arh::stream(stream);
  const size_t bytes = 16 * (size_t)s->nb;
  if (h_pos4) cudaMemcpyAsync(s->pos, h_pos4, bytes, cudaMemcpyHostToDevice, st);
  if (h_quat4) cudaMemcpyAsync(s->quat, h_quat4, bytes, cudaMemcpyHostToDevice, st);
  if (h_vel4) cudaMemcpyAsync(s->vel, h_vel4, bytes, cudaMemcpyHostToDevice, st);
  if (h_ang4) cudaMemcpyAsync(s->ang, h_ang4, bytes, cudaMemcpyHostToDevice, st);
  return arh::check_launch("ar_scene_upload");
}

// The four body-state arrays are adjacent in the scene's block (pos, quat, vel, ang; carved
// 16 * nb bytes apart by alloc_scene_block), so one contiguous copy moves all of them.  A 2D
// copy of the same four rows ran at about 5 GB/s (256 KB each way: 95 us against 12 us).
static_assert(sizeof(float4) == 16, "state rows are 16 * nb bytes");

ar_status ar_scene_upload_state(ar_scene* s, const float* h_state16, ar_stream_t stream) {
  if (!s || !h_state16) return AR_ERR_INVALID_ARG;
  if (s->nb == 0) return AR_OK;
  cudaMemcpyAsync(s->pos, h_state16, 64 * (size_t)s->nb, cudaMemcpyHostToDevice,
                  arh::stream(stream));
  return arh::check_launch("ar_scene_upload_state");
}

ar_status ar_scene_download_state_async(ar_scene* s, float* h_state16, ar_stream_t stream) {
  if (!s || !h_state16) return AR_ERR_INVALID_ARG;
  if (s->nb == 0) return AR_OK;
  cudaMemcpyAsync(h_state16, s->pos, 64 * (size_t)s->nb, cudaMemcpyDeviceToHost,
                  arh::stream(stream));
  return arh::check_launch("ar_scene_download_state_async");
}

ar_status ar_scene_step_io(ar_ctx* ctx, ar_scene* s, const float* h_state_in16, int n_steps,
                           float* h_state_out16, ar_stream_t stream) {
  if (!ctx || !s || !h_state_in16 || !h_state_out16 || n_steps < 0) return AR_ERR_INVALID_ARG;
  ar_status r = ar_scene_upload_state(s, h_state_in16, stream);
  if (r == AR_OK) r = ar_step(ctx, s, n_steps, 1, stream);
  if (r == AR_OK) r = ar_scene_download_state(s, h_state_out16, stream);
  return r;
}

ar_status ar_scene_download_state(ar_scene* s, float* h_state16, ar_stream_t stream) {
  ar_status r = ar_scene_download_state_async(s, h_state16, stream);
  if (r != AR_OK) return r;
  cudaError_t e = cudaStreamSynchronize(arh::stream(stream));
  if (e != cudaSuccess) {
    arh::set_error("ar_scene_download_state: %s", cudaGetErrorString(e));
    return AR_ERR_CUDA;
  }
  return AR_OK;
}

ar_status ar_scene_particle_forces(ar_scene* s, float* p_force4, float* p_torque4,
                                   ar_stream_t stream) {
  (void)p_torque4;
  if (!s || !p_force4 || !s->solo || !s->solo->pforce) return AR_ERR_INVALID_ARG;
  cudaMemcpyAsync(p_force4, s->solo->pforce, 16 * (size_t)s->n, cudaMemcpyDeviceToDevice,
                  arh::stream(stream));
  return arh::check_launch("ar_scene_particle_forces");
}

ar_status ar_scene_step_view(ar_scene* s, ar_step_view* v) {
  if (!s || !v || !s->solo) return AR_ERR_INVALID_ARG;
  ar_batch* B = s->solo;
  const bool bvh = B->broadphase == AR_BROADPHASE_BVH;
  v->num_particles = (int)B->nt;
  v->num_cells = bvh ? 0 : B->total_cells;
  v->key_bits = bvh ? B->bvh_key_bits : B->key_bits;
  const bool k64 = bvh && B->bvh_key_bits > 32;
  v->sorted_keys = k64 ? (uint32_t*)B->skeys64 : B->skeys;
  v->sorted_idx = B->svals;
  v->sorted_pos4 = (float*)B->spos;
  v->sorted_vel4 = (float*)B->svel;
  v->particle_force4 = (float*)B->pforce;
  v->cells2 = bvh ? nullptr : (uint32_t*)B->cells;
  v->key_bytes = k64 ? 8 : 4;
  v->broadphase = B->broadphase;
  v->tree_left = bvh ? B->left : nullptr;
  v->tree_right = bvh ? B->right : nullptr;
  v->tree_parent = bvh ? B->parent : nullptr;
  v->tree_nodes16 = bvh ? (float*)B->nodes : nullptr;
  return AR_OK;
}

ar_status ar_batch_create(ar_ctx* ctx, ar_batch** out) {
  if (!ctx || !out) return AR_ERR_INVALID_ARG;
  ar_batch* B = new ar_batch();
  B->ctx = ctx;
  if (arh::dev_malloc((void**)&B->d_step, sizeof(long long)) != cudaSuccess ||
      cudaMemset(B->d_step, 0, sizeof(long long)) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(B->d_step);
    delete B;
    arh::set_error("ar_batch_create: allocation failed");
    return AR_ERR_OOM;
  }
  *out = B;
  return AR_OK;
}

ar_status ar_batch_destroy(ar_batch* B) {
  if (!B) return AR_ERR_INVALID_ARG;
  cudaDeviceSynchronize();
  drop_graph(B);
  if (B->cap_stream) cudaStreamDestroy(B->cap_stream);
  free_batch_buffers(B);
  cudaFree(B->d_step);
  for (int i = 0; i < 2; ++i) {
    if (B->h_stage[i]) cudaFreeHost(B->h_stage[i]);
    if (B->stage_ev[i]) cudaEventDestroy(B->stage_ev[i]);
  }
  delete B;
  return AR_OK;
}

ar_status ar_batch_set_scenes(ar_batch* B, ar_scene* const* scenes, int n_scenes) {
  if (!B || n_scenes < 0 || (n_scenes > 0 && !scenes)) return AR_ERR_INVALID_ARG;
  for (int i = 0; i < n_scenes; ++i) {
    if (!scenes[i]) return AR_ERR_INVALID_ARG;
    if (scenes[i]->desc.broadphase != scenes[0]->desc.broadphase) {
      arh::set_error("ar_batch_set_scenes: all scenes of a batch use one broad phase");
      return AR_ERR_INVALID_ARG;
    }
  }
  B->scenes.assign(scenes, scenes + n_scenes);
  B->end_steps.clear();
  B->table_dirty = true;
  return AR_OK;
}

ar_status ar_batch_set_scenes_limited(ar_batch* B, ar_scene* const* scenes, int n_scenes,
                                      const int64_t* steps_left) {
  ar_status s = ar_batch_set_scenes(B, scenes, n_scenes);
  if (s != AR_OK || !steps_left) return s;
  B->end_steps.resize(n_scenes);
  for (int i = 0; i < n_scenes; ++i)
    B->end_steps[i] = steps_left[i] < 0 ? LLONG_MAX : B->host_step + steps_left[i];
  return AR_OK;
}

ar_status ar_batch_step(ar_ctx* ctx, ar_batch* B, int n_steps, int use_graph,
                        ar_stream_t stream) {
  if (!ctx || !B || n_steps < 0) return AR_ERR_INVALID_ARG;
  return batch_step(ctx, B, n_steps, use_graph, arh::stream(stream));
}

ar_status ar_batch_model_matrices(ar_batch* B, float* d_model16, ar_stream_t stream) {
  if (!B || !d_model16) return AR_ERR_INVALID_ARG;
  if (((uintptr_t)d_model16 & 15u) != 0) {
    arh::set_error("ar_batch_model_matrices: the output must be 16-byte aligned");
    return AR_ERR_INVALID_ARG;
  }
  cudaStream_t st = arh::stream(stream);
  ar_status s = prepare(B, st);
  if (s != AR_OK) return s;
  if (B->bt == 0) return AR_OK;
  model_matrices_kernel<<<std::min(arh::grid_for(B->bt, 256), 4096u), 256, 0, st>>>(
      B->d_table, B->d_bscene, (int)B->bt, d_model16);
  return arh::check_launch("ar_batch_model_matrices");
}

ar_status ar_scene_model_matrices(ar_scene* s, float* d_model16, ar_stream_t stream) {
  if (!s) return AR_ERR_INVALID_ARG;
  ar_status st = ensure_solo(s);
  if (st != AR_OK) return st;
  return ar_batch_model_matrices(s->solo, d_model16, stream);
}

int ar_batch_launches_per_step(ar_batch* B) {
  if (!B) return 0;
  // BVH: memset, keys, the sort (32-bit keys: memset + four re-sort kernels after the first
  // step; 64-bit keys: the radix sort), three tree kernels (build, leaves + refit, roots),
  // collide, body sums, integration
  if (B->broadphase == AR_BROADPHASE_BVH)
    return 1 + 1 + (B->bvh_key_bits <= 32 ? 1 + 4 : ar_sort::launches(0, B->bvh_key_bits, false)) +
           3 + 1 + 2;
  // a step that re-sorts from the previous order (every step but the first after a change of
  // the member list): clear, keys, four re-sort kernels, scatter, collide (and the static
  // clouds' impulses when a scene has one), body sums, integration
  return 1 /*clear*/ + 1 /*keys*/ + 4 /*re-sort*/ + 1 /*scatter*/ + 1 /*collide*/ +
         (B->has_cloud ? 1 : 0) + 2 /*body sums, integration*/;
}

int ar_scene_launches_per_step(ar_scene* s) {
  if (!s || !s->solo) return 0;
  return ar_batch_launches_per_step(s->solo);
}

}  // extern "C"
