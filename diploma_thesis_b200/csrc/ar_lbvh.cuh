// LBVH device routines shared by the stage entry points (ar_lbvh.cu) and the fused BVH step
// (ar_pipeline.cu): Karras node construction, fenced bottom-up refit, box tests and the
// stackless traversal in the reference's visit order.
//
// Node numbering is the reference's SoA layout (BVHSource/BVHSoAKernels.cu): leaf i at index
// i, internal node i at n + i, root at n.  Boxes are the reference's 32-byte AABB
// {min.xyz, max.xyz, pad, pad}, read as two float4.
#pragma once
#include <cuda/atomic>

#include "ar_internal.cuh"

namespace ar_lbvh {

// ---- longest common prefix (BVHSource/BVHAuxiliary.cuh:31-43) ------------------------------
struct Lcp32 {
  const uint32_t* __restrict__ c;
  int n;
  __device__ __forceinline__ int operator()(int i, int j) const {
    if (j < 0 || j >= n) return -1;
    const uint32_t a = __ldg(c + i), b = __ldg(c + j);
    return a != b ? __clz(a ^ b) : __clz(i ^ j) + 32;
  }
};
struct Lcp64 {
  const uint64_t* __restrict__ c;
  int n;
  __device__ __forceinline__ int operator()(int i, int j) const {
    if (j < 0 || j >= n) return -1;
    const uint64_t a = __ldg((const unsigned long long*)c + i),
                   b = __ldg((const unsigned long long*)c + j);
    return a != b ? __clzll(a ^ b) : __clz(i ^ j) + 64;
  }
};
// 64-bit keys whose top bits (>> shift) name a scene: equal keys are tie-broken by their index
// within the scene, so a scene's subtree is the same as in a tree built over the scene alone.
struct Lcp64Scene {
  const uint64_t* __restrict__ c;
  int n;
  const int* __restrict__ poff;
  int shift;
  __device__ __forceinline__ int operator()(int i, int j) const {
    if (j < 0 || j >= n) return -1;
    const uint64_t a = __ldg((const unsigned long long*)c + i),
                   b = __ldg((const unsigned long long*)c + j);
    if (a != b) return __clzll(a ^ b);
    const int base = __ldg(poff + (int)(a >> shift));
    return __clz((i - base) ^ (j - base)) + 64;
  }
};

// The same for 32-bit keys (scene index above the 30-bit code, at most 4 scenes).  Its
// values are those of Lcp64Scene minus 32 for the same keys, so the topology is the same.
struct Lcp32Scene {
  const uint32_t* __restrict__ c;
  int n;
  const int* __restrict__ poff;
  int shift;
  __device__ __forceinline__ int operator()(int i, int j) const {
    if (j < 0 || j >= n) return -1;
    const uint32_t a = __ldg(c + i), b = __ldg(c + j);
    if (a != b) return __clz(a ^ b);
    const int base = __ldg(poff + (int)(a >> shift));
    return __clz((i - base) ^ (j - base)) + 32;
  }
};

// ---- Karras 2012 internal node i (kernelConstructRadixTreeSoA, BVHSoAKernels.cu:7-99) ----
// Returns the node's (left, right) child ids.
template <class Lcp>
__device__ __forceinline__ int2 karras_node(int i, int n, const Lcp& lcp, uint8_t* is_leaf,
                                            int32_t* left, int32_t* right, int32_t* parent,
                                            int32_t* min_r, int32_t* max_r) {
  const int d = (lcp(i, i + 1) - lcp(i, i - 1)) > 0 ? 1 : -1;
  const int sig_min = lcp(i, i - d);
  int lmax = 2;
  while (lcp(i, i + lmax * d) > sig_min) lmax *= 2;
  int l = 0;
  for (int t = lmax / 2; t >= 1; t /= 2) {
    if (lcp(i, i + (l + t) * d) > sig_min) l += t;
    if (t == 1) break;
  }
  const int j = i + l * d;
  const int sig_node = lcp(i, j);
  // split search: t = ceil(l / 2^k), k = 1, 2, ... (the reference's double division by a
  // power of two is exact, so the integer ceiling is the same value)
  int s = 0;
  for (int k = 1;; ++k) {
    const int t = (int)(((long long)l + (1ll << k) - 1) >> k);
    if (lcp(i, i + (s + t) * d) > sig_node) s += t;
    if (t <= 1) break;
  }
  const int gamma = i + s * d + min(d, 0);
  const int node = n + i;
  const int lo = min(i, j), hi = max(i, j);
  is_leaf[node] = 0;
  const int lc = (lo == gamma) ? gamma : gamma + n;
  const int rc = (hi == gamma + 1) ? gamma + 1 : gamma + 1 + n;
  left[node] = lc;
  right[node] = rc;
  parent[lc] = node;
  parent[rc] = node;
  min_r[node] = lo;
  max_r[node] = hi;
  return make_int2(lc, rc);
}

// ---- bottom-up refit (kernelConstructInternalNodesSoA, BVHSoAKernels.cu:148-176) ------------
// One thread per leaf climbs; the second thread to reach a node merges its children's boxes
// (mergeBounds, BVHAuxiliary.cuh:83-94: min of the mins and max of the maxes, left child
// first) and continues.  The arrival counter is a device-scope acquire-release increment, so
// the first thread's box stores (made before its increment) are visible to the second
// thread's loads (made after it); boxes are read and written through L2.  (Merging the nodes
// inside a block through shared memory instead was measured slower: more dependent loads per
// level outweighed the fences it saved.)
struct Box6 {
  float lx, ly, lz, hx, hy, hz;
};
__device__ __forceinline__ Box6 merge_boxes(const Box6& a, const Box6& b) {  // a = left child
  return Box6{a.lx < b.lx ? a.lx : b.lx, a.ly < b.ly ? a.ly : b.ly, a.lz < b.lz ? a.lz : b.lz,
              a.hx > b.hx ? a.hx : b.hx, a.hy > b.hy ? a.hy : b.hy, a.hz > b.hz ? a.hz : b.hz};
}

// Returns the previous count.
__device__ __forceinline__ int arrive(int* counter) {
  cuda::atomic_ref<int, cuda::thread_scope_device> a(*counter);
  return a.fetch_add(1, cuda::memory_order_acq_rel);
}

// Climb from `leaf`.  `children(node, &left_box, &right_box)` reads both child boxes of
// `node` through L2; `store(node, box)` publishes a node's merged box (before the next
// arrival).  Returns when this thread arrived first or at the root.
template <class Children, class Store>
__device__ __forceinline__ void refit_climb(int leaf, int n, const int32_t* __restrict__ parent,
                                            int* __restrict__ counters, Children children,
                                            Store store) {
  int node = __ldg(parent + leaf);
  for (int depth = 0; depth < n; ++depth) {  // a valid tree is at most n - 1 deep
    if (node < n || node >= 2 * n - 1) return;  // malformed parent link
    if (arrive(counters + (node - n)) == 0) return;
    Box6 a, b;
    children(node, &a, &b);
    store(node, merge_boxes(a, b));
    if (node == n) return;
    node = __ldg(parent + node);
  }
}

// ---- boxes -----------------------------------------------------------------------------------
struct Box {
  float lx, ly, lz, hx, hy, hz;
};
__device__ __forceinline__ Box load_box(const float4* __restrict__ b, int node) {
  const float4 p = __ldg(b + 2 * node), q = __ldg(b + 2 * node + 1);
  return Box{p.x, p.y, p.z, p.w, q.x, q.y};
}
// checkOverlap(AABB, AABB) (BVHAuxiliary.cuh:139-152)
__device__ __forceinline__ bool overlap(const Box& a, const Box& b) {
  return (a.lx <= b.hx && a.hx >= b.lx) && (a.ly <= b.hy && a.hy >= b.ly) &&
         (a.lz <= b.hz && a.hz >= b.lz);
}

// ---- stackless traversal in the reference's order (RB_BVHKernels.cu:145-214) -------------------
// From internal node `root`: at each internal node, the overlapping leaf children are handled
// left then right, then the walk descends into the left internal child if it overlaps, and on
// the way back up into the right one.  visit_leaf(leaf, is_left_child) for every leaf child
// that accept(child) admits.  `root` is never left through its parent link.  A valid tree is
// walked in fewer than 4 (2n - 1) moves; the bound only guards against a malformed tree.
template <class Accept, class Visit>
__device__ __forceinline__ void walk(int root, int n, const uint8_t* __restrict__ is_leaf,
                                     const int32_t* __restrict__ left,
                                     const int32_t* __restrict__ right,
                                     const int32_t* __restrict__ parent, Accept accept,
                                     Visit visit_leaf) {
  int node = root;
  bool descending = true;
  int from = -1;
  for (long moves = 8l * n + 64; moves > 0; --moves) {
    if (descending) {
      const int lc = __ldg(left + node), rc = __ldg(right + node);
      const bool ll = __ldg(is_leaf + lc), rl = __ldg(is_leaf + rc);
      const bool ol = accept(lc), orr = accept(rc);
      if (ol && ll) visit_leaf(lc, true);
      if (orr && rl) visit_leaf(rc, false);
      if (ol && !ll) { node = lc; continue; }
      if (orr && !rl) { node = rc; continue; }
      descending = false;
    } else {
      const int rc = __ldg(right + node);
      if (from == __ldg(left + node) && !__ldg(is_leaf + rc) && accept(rc)) {
        node = rc;
        descending = true;
        continue;
      }
    }
    if (node == root) return;
    from = node;
    node = __ldg(parent + node);
  }
}

}  // namespace ar_lbvh
