// (a9) Karras LBVH hierarchy, (a10) leaves, (a11) bottom-up refit, (a12) traversal.
//
// Node numbering is the reference's SoA layout (BVHSource/BVHSoAKernels.cu): leaf i at index
// i, internal node i at n + i, root at n.  Boxes are the reference's 32-byte AABB
// {min.xyz, max.xyz, pad, pad}, read as two float4.
//
// Traversal is stackless: the tree's parent links replace the reference's int[64] stack.
// The visit order is the reference's (RB_BVHKernels.cu:145-214): at an internal node, its
// overlapping leaf children are handled left then right, then the walk descends into the
// left internal child if it overlaps, and on the way back up into the right one.  Handling
// contacts in the same order keeps the float sums identical to the reference's.
#include <algorithm>

#include "ar_internal.cuh"
#include "ar_dem.cuh"
#include "ar_lbvh.cuh"

using ar_lbvh::Box;
using ar_lbvh::load_box;
using ar_lbvh::overlap;

namespace {

// ---- Karras 2012 internal nodes (kernelConstructRadixTreeSoA, BVHSoAKernels.cu:7-99) -------
template <class Lcp>
__global__ void __launch_bounds__(256) build_kernel(Lcp lcp, int n, uint8_t* __restrict__ is_leaf,
                                                    int32_t* __restrict__ left,
                                                    int32_t* __restrict__ right,
                                                    int32_t* __restrict__ parent,
                                                    int32_t* __restrict__ min_r,
                                                    int32_t* __restrict__ max_r) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) parent[n] = -1;  // root: no parent (the reference leaves it unset)
  if (i >= n - 1) return;
  ar_lbvh::karras_node(i, n, lcp, is_leaf, left, right, parent, min_r, max_r);
}

// ---- leaves (kernelConstructLeafNodesSoA + initializeRadii, BVHSoAKernels.cu:108-138) ------
__global__ void __launch_bounds__(256) leaves_kernel(int n, const int32_t* __restrict__ sorted_idx,
                                                     const float4* __restrict__ pos, float r,
                                                     uint8_t* __restrict__ is_leaf,
                                                     int32_t* __restrict__ min_r,
                                                     int32_t* __restrict__ max_r,
                                                     float4* __restrict__ cms,
                                                     float4* __restrict__ bounds,
                                                     float* __restrict__ radii) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 c = __ldg(pos + __ldg(sorted_idx + i));
  is_leaf[i] = 1;
  min_r[i] = i;
  max_r[i] = i;
  cms[i] = c;
  bounds[2 * i] = make_float4(c.x - r, c.y - r, c.z - r, c.x + r);
  bounds[2 * i + 1] = make_float4(c.y + r, c.z + r, 0.f, 0.f);
  radii[i] = r;
}

// ---- refit (kernelConstructInternalNodesSoA, BVHSoAKernels.cu:148-176) ----------------------
__global__ void __launch_bounds__(256) refit_kernel(int n, const int32_t* __restrict__ left,
                                                    const int32_t* __restrict__ right,
                                                    const int32_t* __restrict__ parent,
                                                    float4* bounds, int* __restrict__ counters) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  auto children = [&](int node, ar_lbvh::Box6* a, ar_lbvh::Box6* b) {
    const int l = __ldg(left + node), r = __ldg(right + node);
    const float4 a0 = __ldcg(bounds + 2 * l), a1 = __ldcg(bounds + 2 * l + 1);
    const float4 b0 = __ldcg(bounds + 2 * r), b1 = __ldcg(bounds + 2 * r + 1);
    *a = ar_lbvh::Box6{a0.x, a0.y, a0.z, a0.w, a1.x, a1.y};
    *b = ar_lbvh::Box6{b0.x, b0.y, b0.z, b0.w, b1.x, b1.y};
  };
  auto store = [&](int node, const ar_lbvh::Box6& m) {
    __stcg(bounds + 2 * node, make_float4(m.lx, m.ly, m.lz, m.hx));
    __stcg(bounds + 2 * node + 1, make_float4(m.hy, m.hz, 0.f, 0.f));
  };
  ar_lbvh::refit_climb(i, n, parent, counters, children, store);
}

// Parent links from the child links, for callers with the reference's traversal signature
// (collideBVHSoARigidBodyWrapper passes no parent array): one thread per internal node.
__global__ void __launch_bounds__(256) parents_kernel(int n, const int32_t* __restrict__ left,
                                                      const int32_t* __restrict__ right,
                                                      int32_t* __restrict__ parent) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const int node = n + i;
  parent[__ldg(left + node)] = node;
  parent[__ldg(right + node)] = node;
  if (i == 0) parent[n] = -1;
}

// ---- collideBVHSoARigidBody (Kernels/RB_BVHKernels.cu:100-244) ------------------------------
__global__ void __launch_bounds__(128) collide_bvh_kernel(
    ar_sim_params prm, const int32_t* __restrict__ rb_idx, const float4* __restrict__ rel,
    const float4* __restrict__ vel, const uint8_t* __restrict__ is_leaf,
    const int32_t* __restrict__ left, const int32_t* __restrict__ right,
    const int32_t* __restrict__ parent, const float4* __restrict__ cms,
    const float4* __restrict__ bounds, const int32_t* __restrict__ sorted_idx,
    const float* __restrict__ radii, int n, float4* __restrict__ p_force,
    float4* __restrict__ p_torque, float4* __restrict__ p_positions) {
  const int index = blockIdx.x * blockDim.x + threadIdx.x;
  if (index >= n) return;
  const int q = __ldg(sorted_idx + index);
  const float3 qvel = ar::xyz(__ldg(vel + q));
  const float4 qpos = __ldg(cms + index);
  const float qrad = __ldg(radii + index);
  const int qbody = __ldg(rb_idx + q);
  const Box qbox = load_box(bounds, index);
  const float4 qrel = __ldg(rel + q);
  const float4 rbcm = make_float4(qpos.x - qrel.x, qpos.y - qrel.y, qpos.z - qrel.z, qpos.w - qrel.w);
  float3 force = ar::mk3(0.f, 0.f, 0.f), torque = ar::mk3(0.f, 0.f, 0.f);
  float4 corr = make_float4(0.f, 0.f, 0.f, 0.f);
  const float3 r3 = ar::xyz(qrel);
  if (n >= 2) {
    ar_lbvh::walk(n, n, is_leaf, left, right, parent,
         [&](int c) { return c != index && overlap(qbox, load_box(bounds, c)); },
         [&](int c, bool is_left) {
           const int oc = __ldg(sorted_idx + c);
           const int ob = __ldg(rb_idx + oc);
           if (!(qbody != ob || qbody == -1)) return;
           float4 lc = make_float4(0.f, 0.f, 0.f, 0.f);
           float3 f = ar_dem::static_pair(qpos, __ldg(cms + c), rbcm, qvel,
                                          ar::xyz(__ldg(vel + oc)), qrad, __ldg(radii + c), prm,
                                          &lc);
           if (!is_left) {  // the right-leaf branch also takes maxOpF4(local, corr) first (:191)
             corr.x = corr.x > lc.x ? corr.x : lc.x;
             corr.y = corr.y > lc.y ? corr.y : lc.y;
             corr.z = corr.z > lc.z ? corr.z : lc.z;
             corr.w = corr.w > lc.w ? corr.w : lc.w;
           }
           corr = make_float4(corr.x + lc.x, corr.y + lc.y, corr.z + lc.z, corr.w + lc.w);
           force = ar::add(force, f);
           torque = ar::add(torque, ar::cross(r3, f));
         });
  }
  if (qbody == -1) return;  // free particles: the reference updates vel in place (not on this path)
  p_force[q] = make_float4(force.x, force.y, force.z, 0.f);
  p_torque[q] = make_float4(torque.x, torque.y, torque.z, 0.f);
  if (p_positions) p_positions[q] = corr;
}

// ---- FindRigidBodyCollisionsBVHKernel (Kernels/RB_BVHKernels.cu:760-876) ---------------------
__global__ void __launch_bounds__(128) find_contacts_kernel(
    const int32_t* __restrict__ rb_idx, const uint8_t* __restrict__ is_leaf,
    const int32_t* __restrict__ left, const int32_t* __restrict__ right,
    const int32_t* __restrict__ parent, const int32_t* __restrict__ max_r,
    const float4* __restrict__ cms, const float4* __restrict__ bounds,
    const int32_t* __restrict__ sorted_idx, const float* __restrict__ radii, int n,
    float* __restrict__ contact_distance, int32_t* __restrict__ colliding_particle,
    int32_t* __restrict__ colliding_body) {
  const int index = blockIdx.x * blockDim.x + threadIdx.x;
  if (index >= n || n < 2) return;
  const int q = __ldg(sorted_idx + index);
  const float4 qpos = __ldg(cms + index);
  const Box qbox = load_box(bounds, index);
  const float qrad = __ldg(radii + q);
  const int qbody = __ldg(rb_idx + q);
  float best = contact_distance[q];
  int best_p = 0, best_b = 0;
  bool found = false;
  ar_lbvh::walk(n, n, is_leaf, left, right, parent,
       [&](int c) {
         return c != index && __ldg(max_r + c) >= index && overlap(qbox, load_box(bounds, c));
       },
       [&](int c, bool) {
         const int oc = __ldg(sorted_idx + c);
         const int ob = __ldg(rb_idx + oc);
         if (qbody == ob) return;
         const float4 cp = __ldg(cms + c);
         const float4 dd = make_float4(cp.x - qpos.x, cp.y - qpos.y, cp.z - qpos.z, cp.w - qpos.w);
         const float dist = sqrtf(dd.x * dd.x + dd.y * dd.y + dd.z * dd.z + dd.w * dd.w);
         const float thr = qrad + __ldg(radii + oc);
         if (thr - dist > best) {
           best = thr - dist;
           best_p = oc;
           best_b = ob;
           found = true;
         }
       });
  if (found) {
    contact_distance[q] = best;
    colliding_particle[q] = best_p;
    colliding_body[q] = best_b;
  }
}

// ---- contact pairs through the BVH ------------------------------------------------------------
__global__ void __launch_bounds__(128) pairs_bvh_kernel(
    float two_r, const int32_t* __restrict__ rb_idx, const uint8_t* __restrict__ is_leaf,
    const int32_t* __restrict__ left, const int32_t* __restrict__ right,
    const int32_t* __restrict__ parent, const float4* __restrict__ cms,
    const float4* __restrict__ bounds, const int32_t* __restrict__ sorted_idx, int n,
    int2* __restrict__ pairs, int capacity, int* __restrict__ count, int* __restrict__ err) {
  const int index = blockIdx.x * blockDim.x + threadIdx.x;
  if (index >= n || n < 2) return;
  const int q = __ldg(sorted_idx + index);
  const float4 qpos = __ldg(cms + index);
  const Box qbox = load_box(bounds, index);
  const int qbody = __ldg(rb_idx + q);
  ar_lbvh::walk(n, n, is_leaf, left, right, parent,
       [&](int c) { return c != index && overlap(qbox, load_box(bounds, c)); },
       [&](int c, bool) {
         if (c < index) return;  // each unordered pair once (from its lower sorted leaf)
         const int oc = __ldg(sorted_idx + c);
         if (__ldg(rb_idx + oc) == qbody) return;
         if (!ar_dem::touching(ar::xyz(qpos), ar::xyz(__ldg(cms + c)), two_r)) return;
         int slot = atomicAdd(count, 1);
         if (slot < capacity)
           pairs[slot] = make_int2(min(q, oc), max(q, oc));
         else
           ar::raise_error(err, ar::kErrOverflow);
       });
}


// ---- static scene through a BVH over its point cloud ----------------------------------------
// checkOverlap(float4, AABB, radius) (BVHSource/BVHAuxiliary.cuh:159-175): the box point
// closest to the sphere centre, distance rounded toward zero, strictly below the radius.
__device__ __forceinline__ bool sphere_box(float4 p, const Box& b, float r) {
  const float xx = fmaxf(b.lx, fminf(p.x, b.hx));
  const float yy = fmaxf(b.ly, fminf(p.y, b.hy));
  const float zz = fmaxf(b.lz, fminf(p.z, b.hz));
  const float d = __fsqrt_rz((xx - p.x) * (xx - p.x) + (yy - p.y) * (yy - p.y) +
                             (zz - p.z) * (zz - p.z));
  return d < r;
}

// staticCollideBVHSoARigidBody (Kernels/RB_BVHKernels.cu:293-442): particle i (unsorted, radius
// params.particle_radius) walks the scene's tree (m leaves) in the reference's order; every
// overlapping leaf adds the DEM force of collideSpheresBVH (BVHAuxiliary.cuh:97-130, the scene
// point at rest) and rel x force.  The reference adds a body's particles' totals straight into
// the body's force and torque with plain read-modify-writes from many threads (racy); here each
// particle's totals go to p_force4 / p_torque4 at its index, for a fixed-order body sum
// (ar_reduce_bodies).  A free particle (body -1) gets v + force as its velocity.  color4 (may
// be NULL): green when a leaf is within touching distance.
__global__ void __launch_bounds__(128) collide_bvh_static_kernel(
    ar_sim_params prm, const int32_t* __restrict__ rb_idx, const float4* __restrict__ rel,
    const float4* __restrict__ pos, float4* __restrict__ vel, const uint8_t* __restrict__ is_leaf,
    const int32_t* __restrict__ left, const int32_t* __restrict__ right,
    const int32_t* __restrict__ parent, const float4* __restrict__ cms,
    const float4* __restrict__ bounds, const float* __restrict__ radii, int m, int n,
    float4* __restrict__ p_force, float4* __restrict__ p_torque, float4* __restrict__ color) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 qpos = __ldg(pos + i);
    const float3 qvel = ar::xyz(vel[i]);
    const float qrad = prm.particle_radius;
    const int qbody = __ldg(rb_idx + i);
    const float3 r3 = ar::xyz(__ldg(rel + i));
    float3 force = ar::mk3(0.f, 0.f, 0.f), torque = force;
    if (m >= 2) {
      ar_lbvh::walk(m, m, is_leaf, left, right, parent,
                    [&](int c) { return sphere_box(qpos, load_box(bounds, c), qrad); },
                    [&](int c, bool) {
                      const float4 cp = __ldg(cms + c);
                      const float rc = __ldg(radii + c);
                      const float3 rp = ar::mk3(cp.x - qpos.x, cp.y - qpos.y, cp.z - qpos.z);
                      const float dist = sqrtf(ar::dot(rp, rp));
                      float3 f = ar::mk3(0.f, 0.f, 0.f);
                      if (dist < qrad + rc)
                        f = ar_dem::spring_force(rp, dist,
                                                 ar::mk3(0.f - qvel.x, 0.f - qvel.y, 0.f - qvel.z),
                                                 qrad + rc, prm.spring, prm.damping, prm.shear,
                                                 prm.attraction);
                      force = ar::add(force, f);
                      torque = ar::add(torque, ar::cross(r3, f));
                      if (dist < qrad + rc && color) color[i] = make_float4(0.f, 1.f, 0.f, 0.f);
                    });
    }
    if (qbody >= 0) {
      p_force[i] = make_float4(force.x, force.y, force.z, 0.f);
      p_torque[i] = make_float4(torque.x, torque.y, torque.z, 0.f);
    } else {
      vel[i] = make_float4(qvel.x + force.x, qvel.y + force.y, qvel.z + force.z, 0.f);
    }
  }
}

// FindAugmentedRealityCollisionsBVHKernel (Kernels/RB_BVHKernels.cu:920-1023): deepest contact
// of particle i with the scene through its tree: an overlapping leaf c (cloud point
// sorted_idx[c]) deepens the contact when r + radii[point] - |cms[c] - p| (four components, as
// the reference's length(float4)) exceeds contact_distance[i], which records it with the point.
// The query radius is params.particle_radius (the reference reads the scene's radius array at
// the query's index; the two agree when every radius is the particle radius).  color4 (may be
// NULL): green on a contact, white when none.
__global__ void __launch_bounds__(128) find_bvh_static_kernel(
    ar_sim_params prm, const float4* __restrict__ pos, const uint8_t* __restrict__ is_leaf,
    const int32_t* __restrict__ left, const int32_t* __restrict__ right,
    const int32_t* __restrict__ parent, const float4* __restrict__ cms,
    const float4* __restrict__ bounds, const int32_t* __restrict__ sorted_idx,
    const float* __restrict__ radii, int m, int n, float* __restrict__ contact_distance,
    int32_t* __restrict__ contact_point, float4* __restrict__ color) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 qpos = __ldg(pos + i);
    const float qrad = prm.particle_radius;
    float deepest = contact_distance[i];
    int best = contact_point[i], ncol = 0;
    if (m >= 2) {
      ar_lbvh::walk(m, m, is_leaf, left, right, parent,
                    [&](int c) { return sphere_box(qpos, load_box(bounds, c), qrad); },
                    [&](int c, bool) {
                      const int s = __ldg(sorted_idx + c);
                      const float4 cp = __ldg(cms + c);
                      const float4 d = make_float4(cp.x - qpos.x, cp.y - qpos.y, cp.z - qpos.z,
                                                   cp.w - qpos.w);
                      const float dist = sqrtf(d.x * d.x + d.y * d.y + d.z * d.z + d.w * d.w);
                      const float thr = qrad + __ldg(radii + s);
                      if (thr - dist > deepest) {
                        ++ncol;
                        deepest = thr - dist;
                        best = s;
                      }
                    });
    }
    contact_distance[i] = deepest;
    contact_point[i] = best;
    if (color) color[i] = ncol ? make_float4(0.f, 1.f, 0.f, 0.f) : make_float4(1.f, 1.f, 1.f, 0.f);
  }
}

// parent links: the caller's, or derived into scratch when the caller has none
const int32_t* parents_or_derive(ar_ctx* ctx, int n, const int32_t* left, const int32_t* right,
                                 const int32_t* parent, cudaStream_t st) {
  if (parent || n < 2) return parent;
  int32_t* p = (int32_t*)arh::scratch(ctx, (size_t)(2 * n - 1) * sizeof(int32_t));
  if (!p) return nullptr;
  parents_kernel<<<arh::grid_for(n - 1, 256), 256, 0, st>>>(n, left, right, p);
  return p;
}

}  // namespace

extern "C" {

ar_status ar_lbvh_build(ar_ctx* ctx, const uint32_t* sorted_codes, int n, uint8_t* is_leaf,
                        int32_t* left, int32_t* right, int32_t* parent, int32_t* min_r,
                        int32_t* max_r, ar_stream_t stream) {
  if (!ctx || n < 0 || (n > 0 && (!sorted_codes || !is_leaf || !left || !right || !parent ||
                                  !min_r || !max_r)))
    return AR_ERR_INVALID_ARG;
  if (n < 2) return AR_OK;
  build_kernel<<<arh::grid_for(n - 1, 256), 256, 0, arh::stream(stream)>>>(
      ar_lbvh::Lcp32{sorted_codes, n}, n, is_leaf, left, right, parent, min_r, max_r);
  return arh::check_launch("ar_lbvh_build");
}

ar_status ar_lbvh_build64(ar_ctx* ctx, const uint64_t* sorted_codes, int n, uint8_t* is_leaf,
                          int32_t* left, int32_t* right, int32_t* parent, int32_t* min_r,
                          int32_t* max_r, ar_stream_t stream) {
  if (!ctx || n < 0 || (n > 0 && (!sorted_codes || !is_leaf || !left || !right || !parent ||
                                  !min_r || !max_r)))
    return AR_ERR_INVALID_ARG;
  if (n < 2) return AR_OK;
  build_kernel<<<arh::grid_for(n - 1, 256), 256, 0, arh::stream(stream)>>>(
      ar_lbvh::Lcp64{sorted_codes, n}, n, is_leaf, left, right, parent, min_r, max_r);
  return arh::check_launch("ar_lbvh_build64");
}

ar_status ar_lbvh_leaves(ar_ctx* ctx, int n, const int32_t* sorted_idx, const float* pos4,
                         float radius, uint8_t* is_leaf, int32_t* min_r, int32_t* max_r,
                         float* cms4, float* bounds8, float* radii, ar_stream_t stream) {
  if (!ctx || n < 0 ||
      (n > 0 && (!sorted_idx || !pos4 || !is_leaf || !min_r || !max_r || !cms4 || !bounds8 ||
                 !radii)))
    return AR_ERR_INVALID_ARG;
  if (n == 0) return AR_OK;
  leaves_kernel<<<arh::grid_for(n, 256), 256, 0, arh::stream(stream)>>>(
      n, sorted_idx, (const float4*)pos4, radius, is_leaf, min_r, max_r, (float4*)cms4,
      (float4*)bounds8, radii);
  return arh::check_launch("ar_lbvh_leaves");
}

ar_status ar_lbvh_refit(ar_ctx* ctx, int n, const int32_t* left, const int32_t* right,
                        const int32_t* parent, float* bounds8, ar_stream_t stream) {
  if (!ctx || n < 0 || (n > 0 && (!left || !right || !parent || !bounds8)))
    return AR_ERR_INVALID_ARG;
  if (n < 2) return AR_OK;
  int* counters = (int*)arh::scratch(ctx, (size_t)(n - 1) * sizeof(int));
  if (!counters) return AR_ERR_OOM;
  cudaStream_t st = arh::stream(stream);
  cudaMemsetAsync(counters, 0, (size_t)(n - 1) * sizeof(int), st);
  refit_kernel<<<arh::grid_for(n, 256), 256, 0, st>>>(n, left, right, parent, (float4*)bounds8,
                                                      counters);
  return arh::check_launch("ar_lbvh_refit");
}

ar_status ar_collide_bvh_dem(ar_ctx* ctx, const ar_sim_params* params, const int32_t* rb_idx,
                             const float* rel4, const float* vel4, const uint8_t* is_leaf,
                             const int32_t* left, const int32_t* right, const int32_t* parent,
                             const float* cms4, const float* bounds8, const int32_t* sorted_idx,
                             const float* radii, int n, float* p_force4, float* p_torque4,
                             float* p_positions4, ar_stream_t stream) {
  if (!ctx || !params || n < 0 ||
      (n > 0 && (!rb_idx || !rel4 || !vel4 || !is_leaf || !left || !right ||
                 !cms4 || !bounds8 || !sorted_idx || !radii || !p_force4 || !p_torque4)))
    return AR_ERR_INVALID_ARG;
  if (n == 0) return AR_OK;
  parent = parents_or_derive(ctx, n, left, right, parent, arh::stream(stream));
  if (!parent && n >= 2) return AR_ERR_OOM;
  collide_bvh_kernel<<<arh::grid_for(n, 128), 128, 0, arh::stream(stream)>>>(
      *params, rb_idx, (const float4*)rel4, (const float4*)vel4, is_leaf, left, right, parent,
      (const float4*)cms4, (const float4*)bounds8, sorted_idx, radii, n, (float4*)p_force4,
      (float4*)p_torque4, (float4*)p_positions4);
  return arh::check_launch("ar_collide_bvh_dem");
}

ar_status ar_collide_bvh_static(ar_ctx* ctx, const ar_sim_params* params, const int32_t* rb_idx,
                                const float* rel4, const float* pos4, float* vel4,
                                const uint8_t* is_leaf, const int32_t* left,
                                const int32_t* right, const int32_t* parent, const float* cms4,
                                const float* bounds8, const float* radii, int num_scene, int n,
                                float* p_force4, float* p_torque4, float* color4,
                                ar_stream_t stream) {
  if (!ctx || !params || n < 0 || num_scene < 0 ||
      (n > 0 && (!rb_idx || !rel4 || !pos4 || !vel4 || !p_force4 || !p_torque4)) ||
      (num_scene >= 2 && (!is_leaf || !left || !right || !cms4 || !bounds8 || !radii)))
    return AR_ERR_INVALID_ARG;
  if (n == 0) return AR_OK;
  cudaStream_t st = arh::stream(stream);
  parent = parents_or_derive(ctx, num_scene, left, right, parent, st);
  if (!parent && num_scene >= 2) return AR_ERR_OOM;
  const unsigned grid = std::min(arh::grid_for(n, 128), (unsigned)ctx->num_sms * 16);
  collide_bvh_static_kernel<<<grid, 128, 0, st>>>(
      *params, rb_idx, (const float4*)rel4, (const float4*)pos4, (float4*)vel4, is_leaf, left,
      right, parent, (const float4*)cms4, (const float4*)bounds8, radii, num_scene, n,
      (float4*)p_force4, (float4*)p_torque4, (float4*)color4);
  return arh::check_launch("ar_collide_bvh_static");
}

ar_status ar_find_contacts_bvh_static(ar_ctx* ctx, const ar_sim_params* params,
                                      const float* pos4, const uint8_t* is_leaf,
                                      const int32_t* left, const int32_t* right,
                                      const int32_t* parent, const float* cms4,
                                      const float* bounds8, const int32_t* sorted_idx,
                                      const float* radii, int num_scene, int n,
                                      float* contact_distance, int32_t* contact_point,
                                      float* color4, ar_stream_t stream) {
  if (!ctx || !params || n < 0 || num_scene < 0 ||
      (n > 0 && (!pos4 || !contact_distance || !contact_point)) ||
      (num_scene >= 2 && (!is_leaf || !left || !right || !cms4 || !bounds8 || !sorted_idx ||
                          !radii)))
    return AR_ERR_INVALID_ARG;
  if (n == 0) return AR_OK;
  cudaStream_t st = arh::stream(stream);
  parent = parents_or_derive(ctx, num_scene, left, right, parent, st);
  if (!parent && num_scene >= 2) return AR_ERR_OOM;
  const unsigned grid = std::min(arh::grid_for(n, 128), (unsigned)ctx->num_sms * 16);
  find_bvh_static_kernel<<<grid, 128, 0, st>>>(
      *params, (const float4*)pos4, is_leaf, left, right, parent, (const float4*)cms4,
      (const float4*)bounds8, sorted_idx, radii, num_scene, n, contact_distance, contact_point,
      (float4*)color4);
  return arh::check_launch("ar_find_contacts_bvh_static");
}

ar_status ar_find_contacts_bvh(ar_ctx* ctx, const int32_t* rb_idx, const uint8_t* is_leaf,
                               const int32_t* left, const int32_t* right, const int32_t* parent,
                               const int32_t* max_r, const float* cms4, const float* bounds8,
                               const int32_t* sorted_idx, const float* radii, int n,
                               float* contact_distance, int32_t* colliding_particle,
                               int32_t* colliding_body, ar_stream_t stream) {
  if (!ctx || n < 0 ||
      (n > 0 && (!rb_idx || !is_leaf || !left || !right || !max_r || !cms4 ||
                 !bounds8 || !sorted_idx || !radii || !contact_distance ||
                 !colliding_particle || !colliding_body)))
    return AR_ERR_INVALID_ARG;
  if (n < 2) return AR_OK;
  parent = parents_or_derive(ctx, n, left, right, parent, arh::stream(stream));
  if (!parent) return AR_ERR_OOM;
  find_contacts_kernel<<<arh::grid_for(n, 128), 128, 0, arh::stream(stream)>>>(
      rb_idx, is_leaf, left, right, parent, max_r, (const float4*)cms4, (const float4*)bounds8,
      sorted_idx, radii, n, contact_distance, colliding_particle, colliding_body);
  return arh::check_launch("ar_find_contacts_bvh");
}

ar_status ar_pairs_bvh(ar_ctx* ctx, float radius, const int32_t* rb_idx, const uint8_t* is_leaf,
                       const int32_t* left, const int32_t* right, const int32_t* parent,
                       const float* cms4, const float* bounds8, const int32_t* sorted_idx, int n,
                       int32_t* pairs2, int capacity, int32_t* d_count, ar_stream_t stream) {
  if (!ctx || n < 0 || capacity < 0 || !d_count ||
      (n > 0 && (!rb_idx || !is_leaf || !left || !right || !cms4 || !bounds8 ||
                 !sorted_idx || (capacity > 0 && !pairs2))))
    return AR_ERR_INVALID_ARG;
  cudaStream_t st = arh::stream(stream);
  cudaMemsetAsync(d_count, 0, sizeof(int32_t), st);
  if (n < 2) return arh::check_launch("ar_pairs_bvh");
  parent = parents_or_derive(ctx, n, left, right, parent, st);
  if (!parent) return AR_ERR_OOM;
  pairs_bvh_kernel<<<arh::grid_for(n, 128), 128, 0, st>>>(
      2.0f * radius, rb_idx, is_leaf, left, right, parent, (const float4*)cms4,
      (const float4*)bounds8, sorted_idx, n, (int2*)pairs2, capacity, d_count, ctx->d_err);
  return arh::check_launch("ar_pairs_bvh");
}

}  // extern "C"
