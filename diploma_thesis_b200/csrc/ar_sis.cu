// The reference's sequential-impulse path (updateUniformGridSIS, RigidBodies/UniformGridUpdate.cpp
// :734-815) on the GPU, in REFERENCE semantics: per-particle deepest contact on the uniform grid,
// the contact list in particle order, and the Gauss-Seidel impulse iterations.  The reference
// runs the last two on the host (Particles/updateFunctions.cpp:1431-1874) with a device round
// trip every step.
//
// The solver is exact, not a parallel approximation.  A contact's update reads and writes only
// the velocities of its (one or two) bodies and its own accumulated impulses, so two contacts
// that share no body commute.  Contacts are therefore given levels -- level(c) = 1 + the highest
// level among earlier contacts on either of its bodies -- and one level at a time is solved in
// parallel: every body sees exactly the sequence of updates of the reference's loop, so the
// results are the reference's bit for bit.  The level assignment is the same in every
// iteration, since it depends only on which bodies each contact touches, and the iterations
// are laid onto one schedule in which each starts before the previous one ends (see the
// schedule notes above sis_levels_kernel).
#include <algorithm>
#include <climits>

#include "ar_glm.cuh"
#include "ar_grid.cuh"
#include "ar_internal.cuh"

namespace {

using ar_glm::cross3;
using ar_glm::dot3;
using ar_glm::mv;

__device__ __forceinline__ float3 f3(float4 a) { return ar::mk3(a.x, a.y, a.z); }
__device__ __forceinline__ float3 add3(float3 a, float3 b) { return ar::add(a, b); }
__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return ar::sub(a, b); }
__device__ __forceinline__ float3 mul3(float s, float3 a) { return ar::mk3(s * a.x, s * a.y, s * a.z); }
// x / y for the solver's updates.  A zero dividend over a finite non-zero divisor gives the
// signed zero that IEEE division gives (sign = sign of x xor sign of y) without dividing;
// bodies at rest make such quotients common, and the shortcut keeps them off the dependent
// chain of the update.  Every other case is the division itself.
__device__ __forceinline__ float qdiv(float x, float y) {
  if (x == 0.f && isfinite(y) && y != 0.f) return signbit(y) ? -x : x;
  return x / y;
}
__device__ __forceinline__ float3 qdiv3(float3 a, float s) {
  return ar::mk3(qdiv(a.x, s), qdiv(a.y, s), qdiv(a.z, s));
}
// glm::normalize(vec3): v * inversesqrt(dot(v, v)), inversesqrt(x) = 1 / sqrt(x)
__device__ __forceinline__ float3 gnormalize(float3 v) {
  const float inv = 1.0f / sqrtf(dot3(v, v));
  return ar::mk3(v.x * inv, v.y * inv, v.z * inv);
}

// ---- FindRigidBodyCollisionsUniformGridKernel (Kernels/RB_UniformGridKernels.cu:731-842) --------
// Per sorted particle: over the 27 neighbour cells (z, y, x = -1..1), occupants of other bodies;
// the deepest penetration 2r - |p - q| above the running maximum (re-read per cell, as the
// reference does) is kept with the other particle's original index and body.
__global__ void __launch_bounds__(128) find_contacts_grid_kernel(
    ar_grid::Grid g, float radius, const int32_t* __restrict__ rb_idx,
    const float4* __restrict__ spos, const uint32_t* __restrict__ gidx,
    const uint32_t* __restrict__ cstart, const uint32_t* __restrict__ cend, int n,
    float* __restrict__ contact_distance, int32_t* __restrict__ colliding_body,
    int32_t* __restrict__ colliding_particle) {
  const int index = blockIdx.x * blockDim.x + threadIdx.x;
  if (index >= n) return;
  const float3 pos = f3(__ldg(spos + index));
  const int3 gp = g.cell_of(pos);
  const uint32_t orig = __ldg(gidx + index);
  const int body = __ldg(rb_idx + orig);
  const float threshold = 2 * radius;
  for (int z = -1; z <= 1; ++z)
    for (int y = -1; y <= 1; ++y)
      for (int x = -1; x <= 1; ++x) {
        const uint32_t h = g.hash(make_int3(gp.x + x, gp.y + y, gp.z + z));
        const uint32_t st = __ldg(cstart + h);
        float best = contact_distance[orig];
        if (st == ar::kEmpty) continue;
        const uint32_t en = __ldg(cend + h);
        for (uint32_t j = st; j < en; ++j) {
          const int o2 = (int)__ldg(gidx + j);
          const int b2 = __ldg(rb_idx + o2);
          if (j == (uint32_t)index || b2 == body) continue;
          const float3 d = sub3(pos, f3(__ldg(spos + j)));
          const float dist = sqrtf(ar::dot(d, d));
          if (threshold - dist > best) {
            best = threshold - dist;
            contact_distance[orig] = best;
            colliding_particle[orig] = o2;
            colliding_body[orig] = b2;
          }
        }
      }
}

// ---- GatherRigidBodyCollisions (Particles/updateFunctions.cpp:1431-1500) -----------------------
// Particles with a contact (distance > 0), in particle order, become contacts: the contact point
// and normal of findExactContactPoint (Particles/CPU_Engine.cpp:461-473, float4 arithmetic with
// helper_math's host normalize, 1 / sqrt), the bias restitution * relative normal velocity, and
// zeroed accumulated impulses.  Order-preserving compaction: per-block counts, their scan, and
// the scatter.
constexpr int kGatherBlock = 256;

__global__ void __launch_bounds__(kGatherBlock) gather_count_kernel(
    const float* __restrict__ contact_distance, int n, int* __restrict__ block_counts) {
  const int i = blockIdx.x * kGatherBlock + threadIdx.x;
  const bool hit = i < n && __ldg(contact_distance + i) > 0.f;
  const int c = __syncthreads_count(hit);
  if (threadIdx.x == 0) block_counts[blockIdx.x] = c;
}

// Exclusive scan of the block counts in one block (any number of blocks, 1024 at a time).
__global__ void __launch_bounds__(1024) gather_scan_kernel(int* __restrict__ block_counts,
                                                           int blocks, int* __restrict__ total) {
  __shared__ int s_warp[32];
  __shared__ int s_carry;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int base = 0; base < blocks; base += 1024) {
    const int i = base + threadIdx.x;
    const int v = i < blocks ? block_counts[i] : 0;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
      int w = s_warp[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      s_warp[lane] = w;
    }
    __syncthreads();
    const int carry = s_carry;
    const int excl = carry + (warp > 0 ? s_warp[warp - 1] : 0) + x - v;
    if (i < blocks) block_counts[i] = excl;
    __syncthreads();
    if (threadIdx.x == 1023) s_carry = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = s_carry;
}

__global__ void __launch_bounds__(kGatherBlock) gather_write_kernel(
    float radius, float restitution, const int32_t* __restrict__ rb_idx,
    const float4* __restrict__ cms, const float4* __restrict__ vel, const float4* __restrict__ ang,
    const float4* __restrict__ rel, const float* __restrict__ contact_distance,
    const int32_t* __restrict__ colliding_body, const int32_t* __restrict__ colliding_particle,
    int n, const int* __restrict__ block_offsets, int capacity, float4* __restrict__ normal,
    float4* __restrict__ point, int32_t* __restrict__ body1, int32_t* __restrict__ body2,
    float* __restrict__ bias, float* __restrict__ acc_impulse, float* __restrict__ acc_friction,
    float* __restrict__ acc_friction2, int* __restrict__ err) {
  __shared__ int s_warp[kGatherBlock / 32];
  const int i = blockIdx.x * kGatherBlock + threadIdx.x;
  const bool hit = i < n && __ldg(contact_distance + i) > 0.f;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t m = __ballot_sync(0xffffffffu, hit);
  if (lane == 0) s_warp[warp] = __popc(m);
  __syncthreads();
  int before = 0;
  for (int w = 0; w < warp; ++w) before += s_warp[w];
  if (!hit) return;
  const int c = block_offsets[blockIdx.x] + before + __popc(m & ((1u << lane) - 1));
  if (c >= capacity) {
    ar::raise_error(err, ar::kErrOverflow);
    return;
  }
  const int b = __ldg(rb_idx + i);
  const int j = __ldg(colliding_particle + i);
  const int b2 = __ldg(colliding_body + i);
  const float4 cm1 = __ldg(cms + b), cm2 = __ldg(cms + b2);
  const float4 r1 = __ldg(rel + i), r2 = __ldg(rel + j);
  const float4 p1 = make_float4(cm1.x + r1.x, cm1.y + r1.y, cm1.z + r1.z, cm1.w + r1.w);
  const float4 p2 = make_float4(cm2.x + r2.x, cm2.y + r2.y, cm2.z + r2.z, cm2.w + r2.w);
  const float t = radius / (radius + radius);
  const float4 cp = make_float4(p1.x + (p2.x - p1.x) * t, p1.y + (p2.y - p1.y) * t,
                                p1.z + (p2.z - p1.z) * t, p1.w + (p2.w - p1.w) * t);
  const float4 d = make_float4(p2.x - p1.x, p2.y - p1.y, p2.z - p1.z, p2.w - p1.w);
  const float inv = 1.0f / sqrtf(d.x * d.x + d.y * d.y + d.z * d.z + d.w * d.w);
  const float4 cn = make_float4(d.x * inv * (-1.f), d.y * inv * (-1.f), d.z * inv * (-1.f),
                                d.w * inv * (-1.f));
  const float3 n3 = f3(cn);
  const float3 v1 = f3(__ldg(vel + b)), w1 = f3(__ldg(ang + b));
  const float3 v2 = f3(__ldg(vel + b2)), w2 = f3(__ldg(ang + b2));
  const float v_rel = ar::dot(add3(v1, ar::cross(w1, f3(r1))), n3) -
                      ar::dot(add3(v2, ar::cross(w2, f3(r2))), n3);
  normal[c] = cn;
  point[c] = cp;
  body1[c] = b;
  body2[c] = b2;
  bias[c] = restitution * v_rel;
  acc_impulse[c] = 0.f;
  acc_friction[c] = 0.f;
  acc_friction2[c] = 0.f;
}

// ---- SequentialImpulseSolver (Particles/updateFunctions.cpp:1580-1874) --------------------------
struct Contacts {
  const float4* normal;
  const float4* point;
  const int32_t* body1;
  const int32_t* body2;
  const float* bias;
  float* acc_impulse;
  float* acc_friction;
  float* acc_friction2;
};
struct Bodies {
  const float4* cms;
  float4* vel;
  float4* ang;
  const float* inv_inertia;  // current (world) inverse inertia, glm::mat3
  const float* mass;
};

__device__ __forceinline__ float clampf(float v, float lo, float hi) {
  return v < lo ? lo : (v > hi ? hi : v);
}

// One contact's update, the reference's loop body.  The reference compares the float values
// with double constants (abs(x) < 0.00001), so the comparisons are made in double here too.
// A contact's geometry: everything in its update that does not depend on the velocities --
// the lever arms, the effective mass mc (set to 1 below 1e-5, as the reference does), the two
// tangent directions and their effective masses, and the friction bound.  It is the same in
// every sweep, so it is computed once, with the reference's expressions, before the sweeps.
struct Geometry {
  float4 g0;  // p1, mc
  float4 g1;  // p2, friction bound
  float4 g2;  // t1, k1
  float4 g3;  // t2, k2
};

__device__ Geometry contact_geometry(float3 n, float4 point, float4 cm1, float4 cm2,
                                     const float* I1, const float* I2, float m1, float m2,
                                     bool two_body, float ar_friction, float rb_friction,
                                     float abs_gravity_y) {
  const float3 p1 = ar::mk3(point.x - cm1.x, point.y - cm1.y, point.z - cm1.z);
  float3 p2 = ar::mk3(0.f, 0.f, 0.f);
  float mc, bound, k1, k2;
  float3 t1 = ar::mk3(1.f, 0.f, 0.f);
  if (!two_body) {
    mc = 1 / m1 + dot3(cross3(mv(I1, cross3(p1, n)), p1), n);
    if ((double)fabsf(mc) < 0.00001) mc = 1.f;
    bound = ar_friction * mc * abs_gravity_y;
    if ((double)fabsf(t1.x - n.x) < 0.0001) t1 = ar::mk3(0.f, 1.f, 0.f);
    else if ((double)fabsf(t1.x + n.x) < 0.0001) t1 = ar::mk3(0.f, 1.f, 0.f);
    t1 = gnormalize(sub3(t1, mul3(dot3(t1, n), n)));
    k1 = 1 / m1 + dot3(cross3(mv(I1, cross3(p1, t1)), p1), t1);
  } else {
    p2 = ar::mk3(point.x - cm2.x, point.y - cm2.y, point.z - cm2.z);
    mc = 1 / m1 + 1 / m2 + dot3(cross3(mv(I1, cross3(p1, n)), p1), n) +
         dot3(cross3(mv(I2, cross3(p2, n)), p2), n);
    if ((double)fabsf(mc) < 0.00001) mc = 1.f;
    bound = rb_friction * mc * abs_gravity_y;
    if ((double)fabsf(t1.x - n.x) < 0.0001) t1 = ar::mk3(0.f, 1.f, 0.f);
    t1 = gnormalize(sub3(t1, mul3(dot3(t1, n), n)));
    k1 = (1 / m1 + dot3(cross3(mv(I1, cross3(p1, t1)), p1), t1)) +
         (1 / m2 + dot3(cross3(mv(I2, cross3(p2, t1)), p2), t1));
  }
  const float3 t2 = gnormalize(cross3(t1, n));
  if (!two_body)
    k2 = 1 / m1 + dot3(cross3(mv(I1, cross3(p1, t2)), p1), t2);
  else
    k2 = (1 / m1 + dot3(cross3(mv(I1, cross3(p1, t2)), p1), t2)) +
         (1 / m2 + dot3(cross3(mv(I2, cross3(p2, t2)), p2), t2));
  return Geometry{make_float4(p1.x, p1.y, p1.z, mc), make_float4(p2.x, p2.y, p2.z, bound),
                  make_float4(t1.x, t1.y, t1.z, k1), make_float4(t2.x, t2.y, t2.z, k2)};
}

// Geometry of every contact (one thread per contact).
__global__ void __launch_bounds__(256) sis_geometry_kernel(
    Contacts C, Bodies B, const int* __restrict__ d_count, int capacity, float ar_friction,
    float rb_friction, float abs_gravity_y, Geometry* __restrict__ geo) {
  const int count = min(*d_count, capacity);
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < count; c += gridDim.x * blockDim.x) {
    const int i1 = C.body1[c], i2 = C.body2[c];
    const bool two = i2 >= 0;
    geo[c] = contact_geometry(f3(C.normal[c]), C.point[c], B.cms[i1],
                              two ? B.cms[i2] : make_float4(0.f, 0.f, 0.f, 0.f),
                              B.inv_inertia + 9 * i1, B.inv_inertia + 9 * (two ? i2 : i1),
                              B.mass[i1], two ? B.mass[i2] : 1.f, two, ar_friction, rb_friction,
                              abs_gravity_y);
  }
}

// A contact in the solver's working order: 11 float4 words -- normal and bias, the four
// geometry words, the two masses and body ids, the two inverse inertias -- stored word-major
// (word k of contact p at k * stride + p), so that a warp loading consecutive contacts reads
// each word as one contiguous run.
constexpr int kRecWords = 11;
__device__ __forceinline__ void pack_contact(const Contacts& C, const Bodies& B,
                                             const Geometry* __restrict__ geo, int c,
                                             float4* __restrict__ out, size_t stride) {
  const int i1 = C.body1[c], i2 = C.body2[c];
  const float4 n = C.normal[c];
  const Geometry g = geo[c];
  float I1[9], I2[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    I1[k] = B.inv_inertia[9 * i1 + k];
    I2[k] = i2 >= 0 ? B.inv_inertia[9 * i2 + k] : 0.f;
  }
  out[0 * stride] = make_float4(n.x, n.y, n.z, C.bias[c]);
  out[1 * stride] = g.g0;
  out[2 * stride] = g.g1;
  out[3 * stride] = g.g2;
  out[4 * stride] = g.g3;
  out[5 * stride] = make_float4(B.mass[i1], i2 >= 0 ? B.mass[i2] : 1.f, __int_as_float(i1),
                       __int_as_float(i2));
  out[6 * stride] = make_float4(I1[0], I1[1], I1[2], I1[3]);
  out[7 * stride] = make_float4(I1[4], I1[5], I1[6], I1[7]);
  out[8 * stride] = make_float4(I1[8], I2[0], I2[1], I2[2]);
  out[9 * stride] = make_float4(I2[3], I2[4], I2[5], I2[6]);
  out[10 * stride] = make_float4(I2[7], I2[8], 0.f, 0.f);
}

// One contact's update: the velocity-dependent part of the reference's loop body.  acc holds
// the accumulated impulse and the two accumulated frictions.
__device__ void solve_packed(const float4* r, float4* acc, const Bodies& B,
                             float upper_bound) {
  const float3 n = f3(r[0]);
  const float bias = r[0].w;
  const float3 p1 = f3(r[1]), t1 = f3(r[3]), t2 = f3(r[4]);
  const float mc = r[1].w, bound = r[2].w, k1 = r[3].w, k2 = r[4].w;
  const float m1 = r[5].x, m2 = r[5].y;
  const int i1 = __float_as_int(r[5].z), i2 = __float_as_int(r[5].w);
  const float I1[9] = {r[6].x, r[6].y, r[6].z, r[6].w, r[7].x, r[7].y, r[7].z, r[7].w, r[8].x};
  const float4 a = *acc;
  float3 v1 = f3(B.vel[i1]), w1 = f3(B.ang[i1]);
  if (i2 == -1) {
    const float3 vel = add3(v1, cross3(w1, p1));
    const float v_rel = dot3(vel, n);
    float corrective = qdiv(-(v_rel + bias), mc);
    const float tmp = clampf(a.x + corrective, 0.f, upper_bound);
    corrective = tmp - a.x;
    float cf1 = qdiv(-dot3(vel, t1), k1);
    const float f1 = clampf(a.y + cf1, -bound, bound);
    cf1 = f1 - a.y;
    float cf2 = qdiv(-dot3(vel, t2), k2);
    const float f2 = clampf(a.z + cf2, -bound, bound);
    cf2 = f2 - a.z;
    *acc = make_float4(tmp, f1, f2, 0.f);
    const float3 imp = add3(add3(mul3(corrective, n), mul3(cf1, t1)), mul3(cf2, t2));
    v1 = add3(v1, qdiv3(imp, m1));
    w1 = add3(w1, mv(I1, cross3(p1, imp)));
    B.vel[i1] = make_float4(v1.x, v1.y, v1.z, 0.f);
    B.ang[i1] = make_float4(w1.x, w1.y, w1.z, 0.f);
    return;
  }
  const float3 p2 = f3(r[2]);
  const float I2[9] = {r[8].y, r[8].z, r[8].w, r[9].x, r[9].y, r[9].z, r[9].w, r[10].x, r[10].y};
  float3 v2 = f3(B.vel[i2]), w2 = f3(B.ang[i2]);
  const float v_rel = dot3(add3(v1, cross3(w1, p1)), n) - dot3(add3(v2, cross3(w2, p2)), n);
  float corrective = qdiv(-(v_rel + bias), mc);
  const float tmp = clampf(a.x + corrective, 0.f, upper_bound);
  corrective = tmp - a.x;
  // friction is accumulated as the reference does, but (as there) not applied between bodies
  const float3 vel = add3(add3(add3(mul3(-1.f, v1), cross3(w1, p1)), v2), cross3(w2, p2));
  *acc = make_float4(tmp, clampf(a.y + qdiv(-dot3(vel, t1), k1), -bound, bound),
                     clampf(a.z + qdiv(-dot3(vel, t2), k2), -bound, bound), 0.f);
  const float3 imp = mul3(corrective, n);
  v1 = add3(v1, qdiv3(imp, m1));
  w1 = add3(w1, mv(I1, cross3(p1, imp)));
  B.vel[i1] = make_float4(v1.x, v1.y, v1.z, 0.f);
  B.ang[i1] = make_float4(w1.x, w1.y, w1.z, 0.f);
  v2 = sub3(v2, qdiv3(imp, m2));
  w2 = sub3(w2, mv(I2, cross3(p2, imp)));
  B.vel[i2] = make_float4(v2.x, v2.y, v2.z, 0.f);
  B.ang[i2] = make_float4(w2.x, w2.y, w2.z, 0.f);
}

constexpr int kSisThreads = 320;   // the sweep block
constexpr int kLevelCap = 8192;    // level runs kept in shared memory up to this many levels
constexpr int kLevelChunk = 2048;  // body pairs staged per step of the level walk
constexpr int kLayoutThreads = 1024;
constexpr size_t kSisSmemMax = 220 * 1024;   // the sweep block's dynamic shared memory
constexpr size_t kWalkSmemMax = 200 * 1024;  // the walk's (its static 16 KB stay below 227 KB)
// The schedule's header in scratch memory: levels, shift, contact count.
enum { kHdrLevels = 0, kHdrShift = 1, kHdrCount = 2, kHdrWords = 4 };

// Schedule.  Each contact gets a level: 1 + the highest level among earlier contacts on either
// of its bodies.  Sweep s solves level b at step b + s * shift of one schedule, where shift
// exceeds the span of levels that any body's contacts cover.  Then no step holds two contacts
// of one body (two items of one step from sweeps s < s' on body x would need levels of x at
// least shift apart), and each body's updates come in the reference's order: within a sweep
// by level, and the last of sweep s (at step <= first + span + s * shift) before the first of
// sweep s + 1.  Every update therefore reads exactly the values the reference's loop gives it,
// while consecutive sweeps overlap.  Step l covers the levels b congruent to l (mod shift)
// with max(1, l - (iterations - 1) shift) <= b <= min(levels, l), so the contacts are packed
// by (level mod shift, level) and each step's contacts are one contiguous run.

// Levels, each body's first and last level, the span and the shift.  The block stages the
// contacts' body pairs in shared memory a chunk at a time and warp 0 walks them in order, a run
// at a time: a run is up to 32 consecutive contacts on one first body A (the gather emits each
// body's contacts together).  Inside a run, with x_j the last level of contact j's other body
// before the run, level_j = 1 + max(level_{j-1}, x_j): A's last level is the previous
// contact's, and an other body met earlier in the same run was last touched at a level no
// higher than level_{j-1}.  Unrolled, level_j = j + 1 + max(last level of A, max_{i<=j}
// (x_i - i)), a prefix maximum over the warp's lanes.  A body's last level is then the level
// of its last contact in the run (atomicMax), its first level the level of its first contact
// when it had none before (atomicMin).  Any order of contacts is walked correctly; short runs
// only leave lanes idle.
// kShared: the walk's last / first levels live in shared memory.
template <bool kShared>
__global__ void __launch_bounds__(256) sis_levels_kernel(
    const int32_t* __restrict__ body1, const int32_t* __restrict__ body2,
    const int* __restrict__ d_count, int capacity, int num_bodies, int* __restrict__ level,
    int* __restrict__ last, int* __restrict__ first, int* __restrict__ hdr,
    int* __restrict__ err) {
  extern __shared__ int s_walk[];
  __shared__ int2 s_pair[kLevelChunk];
  __shared__ int s_span;
  int count = *d_count;
  if (count > capacity) {
    if (threadIdx.x == 0) ar::raise_error(err, ar::kErrOverflow);
    count = capacity;
  }
  int* lastp = kShared ? s_walk : last;
  int* firstp = kShared ? s_walk + num_bodies : first;
  for (int b = threadIdx.x; b < num_bodies; b += blockDim.x) {
    lastp[b] = 0;
    firstp[b] = INT_MAX;
  }
  if (threadIdx.x == 0) s_span = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  int top = 0;
  for (int base = 0; base < count; base += kLevelChunk) {
    const int m = min(kLevelChunk, count - base);
    for (int i = threadIdx.x; i < m; i += blockDim.x)
      s_pair[i] = make_int2(body1[base + i], body2[base + i]);
    __syncthreads();
    if (threadIdx.x < 32) {
      for (int i = 0; i < m;) {  // one run (cut at 32 contacts and at the chunk's end)
        const int j = i + lane;
        const int2 pr = j < m ? s_pair[j] : make_int2(-1, -1);
        const int a = __shfl_sync(0xffffffffu, pr.x, 0);
        const uint32_t off = ~__ballot_sync(0xffffffffu, pr.x == a);
        const int k = off ? __ffs(off) - 1 : 32;  // contacts in the run (lane 0 is one)
        const bool in = lane < k;
        const int b = in && pr.y >= 0 && pr.y != a ? pr.y : -1;  // a self pair touches A only
        const int x = b >= 0 ? lastp[b] : 0;
        const int a_last = lastp[a];
        int y = in ? x - lane : INT_MIN / 2;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const int t = __shfl_up_sync(0xffffffffu, y, d);
          if (lane >= d) y = max(y, t);
        }
        const int l = lane + 1 + max(a_last, y);
        if (in) level[base + j] = l;
        if (b >= 0) {
          atomicMax(lastp + b, l);
          if (x == 0) atomicMin(firstp + b, l);
        }
        const int run_last = __shfl_sync(0xffffffffu, l, k - 1);
        if (lane == 0) {
          lastp[a] = run_last;
          if (a_last == 0) firstp[a] = l;
        }
        top = max(top, run_last);
        i += k;
        __syncwarp();
      }
    }
    __syncthreads();
  }
  int span = 0;
  for (int b = threadIdx.x; b < num_bodies; b += blockDim.x)
    if (firstp[b] != INT_MAX) span = max(span, lastp[b] - firstp[b]);
  atomicMax(&s_span, span);
  __syncthreads();
  if (threadIdx.x == 0) {
    hdr[kHdrLevels] = top;
    hdr[kHdrShift] = max(2, s_span + 1);
    hdr[kHdrCount] = count;
  }
}

// Level sizes (run[l].y, zeroed before).
__global__ void __launch_bounds__(256) sis_sizes_kernel(const int* __restrict__ level,
                                                        const int* __restrict__ hdr,
                                                        int2* __restrict__ run) {
  const int count = hdr[kHdrCount];
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < count; c += gridDim.x * blockDim.x)
    atomicAdd(&run[level[c]].y, 1);
}

// Position of level l in (level mod shift, level) order: class 0 (shift, 2 shift, ...) first,
// then classes 1 .. shift - 1; with levels = Q shift + R, class r >= 1 holds Q + (r <= R)
// levels, so it starts at r Q + min(r - 1, R).
__device__ __forceinline__ int layout_index(int l, int shift, int q, int rem) {
  const int r = l % shift;
  return r == 0 ? l / shift - 1 : r * q + min(r - 1, rem) + (l - r) / shift;
}

// Lays the level runs out: tmp[layout_index(l)] = size of level l, an exclusive scan of tmp,
// then run[l] = (start, start).  tmp holds `levels` ints.
__global__ void __launch_bounds__(kLayoutThreads) sis_layout_kernel(const int* __restrict__ hdr,
                                                                    int2* __restrict__ run,
                                                                    int* __restrict__ tmp) {
  __shared__ int s_warp[kLayoutThreads / 32];
  __shared__ int s_carry;
  const int levels = hdr[kHdrLevels], shift = hdr[kHdrShift];
  const int q = levels / shift, rem = levels % shift;
  for (int l = 1 + threadIdx.x; l <= levels; l += blockDim.x)
    tmp[layout_index(l, shift, q, rem)] = run[l].y;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int base = 0; base < levels; base += blockDim.x) {
    const int j = base + threadIdx.x;
    const int v = j < levels ? tmp[j] : 0;
    int x = v;  // inclusive warp scan
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, d);
      if (lane >= d) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
      int w = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : 0;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, w, d);
        if (lane >= d) w += y;
      }
      s_warp[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    const int carry = s_carry;
    const int excl = carry + (warp > 0 ? s_warp[warp - 1] : 0) + x - v;
    if (j < levels) tmp[j] = excl;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) s_carry = excl + v;
    __syncthreads();
  }
  for (int l = 1 + threadIdx.x; l <= levels; l += blockDim.x) {
    const int start = tmp[layout_index(l, shift, q, rem)];
    run[l] = make_int2(start, start);
  }
}

// Each contact takes the next slot of its level's run (the order inside a level is free: its
// contacts share no body) and is packed there with its accumulators; order[p] = contact.
// Afterwards level l occupies [run[l].y, run[l].x).
__global__ void __launch_bounds__(256) sis_pack_kernel(Contacts C, Bodies B,
                                                       const Geometry* __restrict__ geo,
                                                       const int* __restrict__ level,
                                                       const int* __restrict__ hdr,
                                                       int capacity, int2* __restrict__ run,
                                                       int* __restrict__ order,
                                                       float4* __restrict__ rec,
                                                       float4* __restrict__ accs) {
  const int count = hdr[kHdrCount];
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < count; c += gridDim.x * blockDim.x) {
    const int p = atomicAdd(&run[level[c]].x, 1);
    order[p] = c;
    pack_contact(C, B, geo, c, rec + p, (size_t)capacity);
    accs[p] = make_float4(C.acc_impulse[c], C.acc_friction[c], C.acc_friction2[c], 0.f);
  }
}

// The accumulated impulses back to the caller's arrays, in contact order.
__global__ void __launch_bounds__(256) sis_writeback_kernel(Contacts C,
                                                            const int* __restrict__ hdr,
                                                            const int* __restrict__ order,
                                                            const float4* __restrict__ accs) {
  const int count = hdr[kHdrCount];
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < count; p += gridDim.x * blockDim.x) {
    const int c = order[p];
    const float4 a = accs[p];
    C.acc_impulse[c] = a.x;
    C.acc_friction[c] = a.y;
    C.acc_friction2[c] = a.z;
  }
}

// A packed contact and its accumulators, held in registers.
struct Item {
  float4 r[kRecWords];
  float4 acc;
  int p;  // packed index, -1: none
};

__device__ __forceinline__ void load_item(const float4* rec, size_t stride, const float4* accs,
                                          int p, Item& it) {
  it.p = p;
  if (p < 0) return;
#pragma unroll
  for (int k = 0; k < kRecWords; ++k) it.r[k] = __ldcg(rec + k * stride + p);
  it.acc = __ldcg(accs + p);
}

// The per-sweep levels lo, lo + shift, ..., hi that one step of the schedule covers, advanced
// one step at a time without division.
struct StepRange {
  int lo, hi;  // the step has contacts while lo <= hi
  int step;
  __device__ void advance(int levels, int iterations, int shift) {
    ++step;
    // the largest level <= min(step, levels) congruent to step
    if (++hi > levels) hi -= shift;
    // the smallest level >= max(1, step - (iterations - 1) shift) congruent to step
    if (step - 1 < iterations * shift) {
      if (++lo > shift) lo -= shift;
    } else {
      ++lo;
    }
  }
};

// The sweeps, in one block: the steps are solved in order with a barrier between them; each
// thread loads its item of the next step (record and accumulators, from L2) while it solves
// the current one, which is safe because an item's accumulators were last written
// shift >= 2 steps earlier.  kShared: the bodies' velocities and angular velocities live in
// shared memory.
template <bool kShared>
__global__ void __launch_bounds__(kSisThreads) sis_sweep_kernel(
    Bodies B, const int* __restrict__ hdr, int capacity, int num_bodies, int iterations,
    float upper_bound, const int2* __restrict__ run, const float4* __restrict__ rec,
    float4* __restrict__ accs) {
  // (kShared) vel[num_bodies], ang[num_bodies], then the level runs when they fit
  extern __shared__ float4 s_mem[];
  const int levels = hdr[kHdrLevels], shift = hdr[kHdrShift];
  float4* s_bodies = s_mem;
  int2* s_run = reinterpret_cast<int2*>(s_bodies + (kShared ? 2 * num_bodies : 0));
  Bodies W = B;
  const int2* runs = run;
  if (levels + 1 <= kLevelCap) {
    for (int l = threadIdx.x; l <= levels; l += blockDim.x) s_run[l] = run[l];
    runs = s_run;
  }
  if (kShared) {
    for (int b = threadIdx.x; b < num_bodies; b += blockDim.x) {
      s_bodies[b] = B.vel[b];
      s_bodies[num_bodies + b] = B.ang[b];
    }
    W.vel = s_bodies;
    W.ang = s_bodies + num_bodies;
  }
  __syncthreads();
  if (levels > 0) {
    const int steps = levels + (iterations - 1) * shift;  // fits in int: checked by the host
    StepRange nr{1, 1, 1};  // step 1 covers level 1 of sweep 0 only
    int next_lo = runs[1].y, next_hi = runs[1].x;
    Item nxt;
    load_item(rec, capacity, accs,
              next_lo + (int)threadIdx.x < next_hi ? next_lo + (int)threadIdx.x : -1, nxt);
    for (int step = 1; step <= steps; ++step) {
      const Item cur = nxt;
      const int lo = next_lo, hi = next_hi;
      if (step < steps) {
        nr.advance(levels, iterations, shift);
        next_lo = next_hi = 0;
        if (nr.lo <= nr.hi) {
          next_lo = runs[nr.lo].y;
          next_hi = runs[nr.hi].x;
        }
        const int p = next_lo + (int)threadIdx.x;
        load_item(rec, capacity, accs, p < next_hi ? p : -1, nxt);
      }
      if (cur.p >= 0) {
        float4 a = cur.acc;
        solve_packed(cur.r, &a, W, upper_bound);
        accs[cur.p] = a;
        // items beyond one per thread
        for (int p = lo + (int)(threadIdx.x + blockDim.x); p < hi; p += blockDim.x) {
          Item more;
          load_item(rec, capacity, accs, p, more);
          a = more.acc;
          solve_packed(more.r, &a, W, upper_bound);
          accs[p] = a;
        }
      }
      __syncthreads();
    }
  }
  if (kShared) {
    for (int b = threadIdx.x; b < num_bodies; b += blockDim.x) {
      B.vel[b] = W.vel[b];
      B.ang[b] = W.ang[b];
    }
  }
}

}  // namespace

extern "C" {

ar_status ar_find_contacts_grid(ar_ctx* ctx, const ar_sim_params* params, const int32_t* rb_idx,
                                const float* sorted_pos4, const uint32_t* grid_idx,
                                const uint32_t* cell_start, const uint32_t* cell_end, int n,
                                float* contact_distance, int32_t* colliding_body,
                                int32_t* colliding_particle, ar_stream_t stream) {
  if (!ctx || !params || n < 0 ||
      (n > 0 && (!rb_idx || !sorted_pos4 || !grid_idx || !cell_start || !cell_end ||
                 !contact_distance || !colliding_body || !colliding_particle)))
    return AR_ERR_INVALID_ARG;
  for (int a = 0; a < 3; ++a) {
    const uint32_t g = params->grid_size[a];
    if (!g || (g & (g - 1))) {
      arh::set_error("grid_size must be powers of two (the hash wraps with & (G-1))");
      return AR_ERR_INVALID_ARG;
    }
  }
  if (n == 0) return AR_OK;
  find_contacts_grid_kernel<<<arh::grid_for(n, 128), 128, 0, arh::stream(stream)>>>(
      ar_grid::Grid::from_params(*params), params->particle_radius, rb_idx,
      (const float4*)sorted_pos4, grid_idx, cell_start, cell_end, n, contact_distance,
      colliding_body, colliding_particle);
  return arh::check_launch("ar_find_contacts_grid");
}

ar_status ar_gather_contacts(ar_ctx* ctx, const ar_sim_params* params, int n,
                             const int32_t* rb_idx, const float* cms4, const float* vel4,
                             const float* ang4, const float* rel4, const float* contact_distance,
                             const int32_t* colliding_body, const int32_t* colliding_particle,
                             int capacity, float* normal4, float* point4, int32_t* body1,
                             int32_t* body2, float* bias, float* acc_impulse,
                             float* acc_friction, float* acc_friction2, int32_t* d_count,
                             ar_stream_t stream) {
  if (!ctx || !params || n < 0 || capacity < 0 || !d_count ||
      (n > 0 && (!rb_idx || !cms4 || !vel4 || !ang4 || !rel4 || !contact_distance ||
                 !colliding_body || !colliding_particle)) ||
      (capacity > 0 && (!normal4 || !point4 || !body1 || !body2 || !bias || !acc_impulse ||
                        !acc_friction || !acc_friction2)))
    return AR_ERR_INVALID_ARG;
  cudaStream_t st = arh::stream(stream);
  if (n == 0) {
    cudaMemsetAsync(d_count, 0, sizeof(int32_t), st);
    return arh::check_launch("ar_gather_contacts");
  }
  const int blocks = (int)arh::grid_for(n, kGatherBlock);
  int* offsets = (int*)arh::scratch(ctx, sizeof(int) * (size_t)blocks);
  if (!offsets) return AR_ERR_OOM;
  gather_count_kernel<<<blocks, kGatherBlock, 0, st>>>(contact_distance, n, offsets);
  gather_scan_kernel<<<1, 1024, 0, st>>>(offsets, blocks, d_count);
  gather_write_kernel<<<blocks, kGatherBlock, 0, st>>>(
      params->particle_radius, params->rb_restitution, rb_idx, (const float4*)cms4,
      (const float4*)vel4, (const float4*)ang4, (const float4*)rel4, contact_distance,
      colliding_body, colliding_particle, n, offsets, capacity, (float4*)normal4,
      (float4*)point4, body1, body2, bias, acc_impulse, acc_friction, acc_friction2, ctx->d_err);
  return arh::check_launch("ar_gather_contacts");
}

ar_status ar_sequential_impulse(ar_ctx* ctx, const ar_sim_params* params, const int32_t* d_count,
                                int capacity, const float* normal4, const float* point4,
                                const int32_t* body1, const int32_t* body2, const float* bias,
                                float* acc_impulse, float* acc_friction, float* acc_friction2,
                                int num_bodies, const float* cms4, float* vel4, float* ang4,
                                const float* cur_inv_inertia9, const float* mass, int iterations,
                                ar_stream_t stream) {
  if (!ctx || !params || !d_count || capacity < 0 || num_bodies < 0 || iterations < 0 ||
      (capacity > 0 && (!normal4 || !point4 || !body1 || !body2 || !bias || !acc_impulse ||
                        !acc_friction || !acc_friction2)) ||
      (num_bodies > 0 && (!cms4 || !vel4 || !ang4 || !cur_inv_inertia9 || !mass)))
    return AR_ERR_INVALID_ARG;
  if (capacity == 0 || num_bodies == 0 || iterations == 0) return AR_OK;
  // the schedule has at most capacity + (iterations - 1) (capacity + 1) steps, counted in int
  if ((long long)iterations * ((long long)capacity + 1) > INT_MAX) {
    arh::set_error("iterations x (capacity + 1) must stay below 2^31");
    return AR_ERR_INVALID_ARG;
  }
  // scratch: geometry[capacity] (64-byte aligned), records (word-major) and accumulators,
  // level runs run[capacity + 1], the schedule header, then level[capacity], order[capacity],
  // last[num_bodies], first[num_bodies]
  const size_t geo_bytes = sizeof(Geometry) * (size_t)capacity;
  const size_t rec_bytes = sizeof(float4) * (size_t)capacity * (kRecWords + 1);
  const size_t run_bytes = sizeof(int2) * ((size_t)capacity + 1);
  const size_t words = kHdrWords + 2 * (size_t)capacity + 2 * (size_t)num_bodies;
  char* base = (char*)arh::scratch(ctx, geo_bytes + rec_bytes + run_bytes + sizeof(int) * words);
  if (!base) return AR_ERR_OOM;
  Geometry* geo = (Geometry*)base;
  float4* rec = (float4*)(base + geo_bytes);
  float4* accs = rec + (size_t)capacity * kRecWords;
  int2* run = (int2*)(base + geo_bytes + rec_bytes);
  int* hdr = (int*)(base + geo_bytes + rec_bytes + run_bytes);
  int* level = hdr + kHdrWords;
  int* order = level + capacity;
  int* last = order + capacity;
  int* first = last + num_bodies;
  Contacts C{(const float4*)normal4, (const float4*)point4, body1, body2, bias, acc_impulse,
             acc_friction, acc_friction2};
  Bodies B{(const float4*)cms4, (float4*)vel4, (float4*)ang4, cur_inv_inertia9, mass};
  cudaStream_t st = arh::stream(stream);
  const unsigned gg = std::min(arh::grid_for(capacity, 256), (unsigned)ctx->num_sms * 8);
  sis_geometry_kernel<<<gg, 256, 0, st>>>(C, B, d_count, capacity, params->ar_friction,
                                          params->rb_friction, fabsf(params->gravity[1]), geo);
  cudaMemsetAsync(run, 0, run_bytes, st);
  // levels: the walk's last / first levels in shared memory when they fit
  const size_t walk_smem = 8 * (size_t)num_bodies;
  if (walk_smem <= kWalkSmemMax) {
    cudaFuncSetAttribute(sis_levels_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)walk_smem);
    sis_levels_kernel<true><<<1, 256, walk_smem, st>>>(body1, body2, d_count, capacity,
                                                      num_bodies, level, last, first, hdr,
                                                      ctx->d_err);
  } else {
    sis_levels_kernel<false><<<1, 256, 0, st>>>(body1, body2, d_count, capacity, num_bodies,
                                               level, last, first, hdr, ctx->d_err);
  }
  sis_sizes_kernel<<<gg, 256, 0, st>>>(level, hdr, run);
  sis_layout_kernel<<<1, kLayoutThreads, 0, st>>>(hdr, run, order);
  sis_pack_kernel<<<gg, 256, 0, st>>>(C, B, geo, level, hdr, capacity, run, order, rec, accs);
  // sweeps: level runs in shared memory; the bodies' velocities too when they fit
  const size_t base_smem = sizeof(int2) * (size_t)kLevelCap;
  const size_t smem = base_smem + 32 * (size_t)num_bodies;
  if (smem <= kSisSmemMax) {
    cudaFuncSetAttribute(sis_sweep_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
    sis_sweep_kernel<true><<<1, kSisThreads, smem, st>>>(B, hdr, capacity, num_bodies,
                                                         iterations, 100.f, run, rec, accs);
  } else {
    cudaFuncSetAttribute(sis_sweep_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)base_smem);
    sis_sweep_kernel<false><<<1, kSisThreads, base_smem, st>>>(B, hdr, capacity, num_bodies,
                                                               iterations, 100.f, run, rec,
                                                               accs);
  }
  sis_writeback_kernel<<<gg, 256, 0, st>>>(C, hdr, order, accs);
  return arh::check_launch("ar_sequential_impulse");
}

}  // extern "C"
