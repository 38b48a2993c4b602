/*
 * oracle.c -- CPU restatement of AR_Sim's per-step rigid-body path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker: tests/, bench.py's cpu_baseline / reference
 * arm and __graft_entry__.smoke() call it to verify (or time a CPU baseline against) the CUDA
 * library; the product never links or calls it.
 *
 * Parity is pinned two ways: the float32 functions here are checked against golden vectors
 * produced by the reference's own kernel bodies run on the CPU (oracle/ref_build.py,
 * tests/golden/make_golden.py), and the CUDA kernels are checked against these functions.
 *
 * Build: gcc -O2 -fPIC -shared -fopenmp -ffp-contract=off (no FMA contraction, SSE float
 * arithmetic), so every float expression is rounded exactly as written -- the same rounding
 * the CUDA library gets from -fmad=false.  Functions whose name ends in _f64 restate the
 * physics in double precision (the FP64 oracle).
 *
 * Each function cites the reference file:line (within AR_Sim/) whose algorithm it follows.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define EMPTY 0xffffffffu

typedef struct { float x, y, z; } v3;
typedef struct { float x, y, z, w; } v4;
typedef struct { double x, y, z; } d3;
typedef struct { double x, y, z, w; } d4;

static inline v3 mk3(float x, float y, float z) { v3 r = {x, y, z}; return r; }
static inline v3 xyz(const float* p) { return mk3(p[0], p[1], p[2]); }
static inline v3 add(v3 a, v3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 sub(v3 a, v3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 scl(float s, v3 a) { return mk3(s * a.x, s * a.y, s * a.z); }
static inline float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 cross(v3 a, v3 b) {
  return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline v3 divs(v3 a, float s) { return mk3(a.x / s, a.y / s, a.z / s); }
static inline v4 ld4(const float* p) { v4 r = {p[0], p[1], p[2], p[3]}; return r; }
static inline void st4(float* p, float x, float y, float z, float w) {
  p[0] = x; p[1] = y; p[2] = z; p[3] = w;
}
static inline int f2i(float f) { int i; memcpy(&i, &f, 4); return i; }
static inline float i2f(int i) { float f; memcpy(&f, &i, 4); return f; }

/* unit quaternion (x, y, z, w) rotation: t = 2 (u x v); v + w t + u x t */
static inline v3 quat_rotate(v4 q, v3 v) {
  v3 u = mk3(q.x, q.y, q.z);
  v3 t = scl(2.0f, cross(u, v));
  return add(add(v, scl(q.w, t)), cross(u, t));
}

/* glm 0.9.7 operations (Libs/glm/glm/detail/type_mat3x3.inl:501-548, gtc/quaternion.inl) */
static inline v3 glm_mv(const float* m, v3 v) {
  return mk3(m[0] * v.x + m[3] * v.y + m[6] * v.z, m[1] * v.x + m[4] * v.y + m[7] * v.z,
             m[2] * v.x + m[5] * v.y + m[8] * v.z);
}
static inline v3 glm_cross(v3 x, v3 y) {
  return mk3(x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y);
}
static void glm_mm(const float* a, const float* b, float* r) {
  for (int c = 0; c < 3; ++c)
    for (int rr = 0; rr < 3; ++rr)
      r[c * 3 + rr] = a[0 * 3 + rr] * b[c * 3 + 0] + a[1 * 3 + rr] * b[c * 3 + 1] +
                      a[2 * 3 + rr] * b[c * 3 + 2];
}
static void glm_mat3_cast(v4 q, float* m) {
  float qxx = q.x * q.x, qyy = q.y * q.y, qzz = q.z * q.z;
  float qxz = q.x * q.z, qxy = q.x * q.y, qyz = q.y * q.z;
  float qwx = q.w * q.x, qwy = q.w * q.y, qwz = q.w * q.z;
  m[0] = 1 - 2 * (qyy + qzz); m[1] = 2 * (qxy + qwz); m[2] = 2 * (qxz - qwy);
  m[3] = 2 * (qxy - qwz); m[4] = 1 - 2 * (qxx + qzz); m[5] = 2 * (qyz + qwx);
  m[6] = 2 * (qxz + qwy); m[7] = 2 * (qyz - qwx); m[8] = 1 - 2 * (qxx + qyy);
}
static v4 glm_qnormalize(v4 q) {
  float len = sqrtf((q.x * q.x + q.y * q.y) + (q.z * q.z + q.w * q.w));
  v4 r = {0.f, 0.f, 0.f, 1.f};
  if (len <= 0.f) return r;
  float inv = 1.f / len;
  r.x = q.x * inv; r.y = q.y * inv; r.z = q.z * inv; r.w = q.w * inv;
  return r;
}
static v4 glm_qmul(v4 p, v4 q) {
  v4 r;
  r.w = p.w * q.w - p.x * q.x - p.y * q.y - p.z * q.z;
  r.x = p.w * q.x + p.x * q.w + p.y * q.z - p.z * q.y;
  r.y = p.w * q.y + p.y * q.w + p.z * q.x - p.x * q.z;
  r.z = p.w * q.z + p.z * q.w + p.x * q.y - p.y * q.x;
  return r;
}

/* ====================================================================================
 * (a6) scene AABB -- findAABBCub (BVHSource/createMortonCodes.cu:65-107)
 * ==================================================================================== */
void or_aabb(const float* pos4, long n, float* mn4, float* mx4) {
  for (int c = 0; c < 4; ++c) { mn4[c] = 2139095040.0f; mx4[c] = -2139095040.0f; }
  for (long i = 0; i < n; ++i)
    for (int c = 0; c < 4; ++c) {
      float v = pos4[4 * i + c];
      if (v < mn4[c]) mn4[c] = v;
      if (v > mx4[c]) mx4[c] = v;
    }
}

/* ====================================================================================
 * (a7) Morton codes -- morton3D / generateMortonCodes (BVHSource/BVHkernels.cu:646-716).
 * The interleave is done bit by bit (an independent check of the multiply-and-mask form).
 * ==================================================================================== */
static uint32_t quantise(float x, float scale, float top) {
  float v = fminf(fmaxf(x * scale, 0.0f), top);
  return (uint32_t)v;
}
void or_morton30(const float* pos4, long n, const float* mn4, const float* mx4, uint32_t* codes) {
  float ex = mx4[0] - mn4[0], ey = mx4[1] - mn4[1], ez = mx4[2] - mn4[2];
  for (long i = 0; i < n; ++i) {
    uint32_t q[3];
    q[0] = quantise((pos4[4 * i + 0] - mn4[0]) / ex, 1024.0f, 1023.0f);
    q[1] = quantise((pos4[4 * i + 1] - mn4[1]) / ey, 1024.0f, 1023.0f);
    q[2] = quantise((pos4[4 * i + 2] - mn4[2]) / ez, 1024.0f, 1023.0f);
    uint32_t c = 0;
    for (int b = 0; b < 10; ++b)
      c |= (((q[0] >> b) & 1u) << (3 * b + 2)) | (((q[1] >> b) & 1u) << (3 * b + 1)) |
           (((q[2] >> b) & 1u) << (3 * b));
    codes[i] = c;
  }
}
void or_morton63(const float* pos4, long n, const float* mn4, const float* mx4, uint64_t* codes) {
  float ex = mx4[0] - mn4[0], ey = mx4[1] - mn4[1], ez = mx4[2] - mn4[2];
  for (long i = 0; i < n; ++i) {
    uint64_t q[3];
    q[0] = quantise((pos4[4 * i + 0] - mn4[0]) / ex, 2097152.0f, 2097151.0f);
    q[1] = quantise((pos4[4 * i + 1] - mn4[1]) / ey, 2097152.0f, 2097151.0f);
    q[2] = quantise((pos4[4 * i + 2] - mn4[2]) / ez, 2097152.0f, 2097151.0f);
    uint64_t c = 0;
    for (int b = 0; b < 21; ++b)
      c |= (((q[0] >> b) & 1ull) << (3 * b + 2)) | (((q[1] >> b) & 1ull) << (3 * b + 1)) |
           (((q[2] >> b) & 1ull) << (3 * b));
    codes[i] = c;
  }
}

/* ====================================================================================
 * (a8) stable sort by key -- cub::DeviceRadixSort::SortPairs semantics: keys ascending,
 * equal keys in input order.  Values permuted along (val == NULL: identity).
 * ==================================================================================== */
static void lsd_sort_u64(uint64_t* keys, uint32_t* vals, long n, int key_bits) {
  uint64_t* k2 = (uint64_t*)malloc(sizeof(uint64_t) * (n ? n : 1));
  uint32_t* v2 = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  uint64_t* ka = keys; uint32_t* va = vals; uint64_t* kb = k2; uint32_t* vb = v2;
  for (int shift = 0; shift < key_bits; shift += 8) {
    long cnt[257];
    memset(cnt, 0, sizeof(cnt));
    for (long i = 0; i < n; ++i) cnt[((ka[i] >> shift) & 0xff) + 1]++;
    for (int d = 0; d < 256; ++d) cnt[d + 1] += cnt[d];
    for (long i = 0; i < n; ++i) {
      long dst = cnt[(ka[i] >> shift) & 0xff]++;
      kb[dst] = ka[i];
      vb[dst] = va[i];
    }
    uint64_t* tk = ka; ka = kb; kb = tk;
    uint32_t* tv = va; va = vb; vb = tv;
  }
  if (ka != keys) {
    memcpy(keys, ka, sizeof(uint64_t) * n);
    memcpy(vals, va, sizeof(uint32_t) * n);
  }
  free(k2);
  free(v2);
}
void or_sort_pairs_u32(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                       uint32_t* vals_out, long n, int begin_bit, int end_bit) {
  uint64_t* k = (uint64_t*)malloc(sizeof(uint64_t) * (n ? n : 1));
  uint64_t mask = end_bit - begin_bit >= 64 ? ~0ull : ((1ull << (end_bit - begin_bit)) - 1);
  for (long i = 0; i < n; ++i) {
    k[i] = ((uint64_t)keys_in[i] >> begin_bit) & mask;
    vals_out[i] = vals_in ? vals_in[i] : (uint32_t)i;
  }
  /* sort (digit, original position) then gather */
  uint32_t* pos = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  for (long i = 0; i < n; ++i) pos[i] = (uint32_t)i;
  lsd_sort_u64(k, pos, n, end_bit - begin_bit);
  uint32_t* tmpv = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  for (long i = 0; i < n; ++i) {
    keys_out[i] = keys_in[pos[i]];
    tmpv[i] = vals_in ? vals_in[pos[i]] : pos[i];
  }
  memcpy(vals_out, tmpv, sizeof(uint32_t) * n);
  free(k); free(pos); free(tmpv);
}
void or_sort_pairs_u64(const uint64_t* keys_in, const uint32_t* vals_in, uint64_t* keys_out,
                       uint32_t* vals_out, long n, int begin_bit, int end_bit) {
  uint64_t* k = (uint64_t*)malloc(sizeof(uint64_t) * (n ? n : 1));
  uint64_t mask = end_bit - begin_bit >= 64 ? ~0ull : ((1ull << (end_bit - begin_bit)) - 1);
  uint32_t* pos = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  for (long i = 0; i < n; ++i) { k[i] = (keys_in[i] >> begin_bit) & mask; pos[i] = (uint32_t)i; }
  lsd_sort_u64(k, pos, n, end_bit - begin_bit);
  for (long i = 0; i < n; ++i) {
    keys_out[i] = keys_in[pos[i]];
    vals_out[i] = vals_in ? vals_in[pos[i]] : pos[i];
  }
  free(k); free(pos);
}

/* ====================================================================================
 * (a9) Karras 2012 radix tree -- kernelConstructRadixTreeSoA (BVHSource/BVHSoAKernels.cu:7-99)
 * with longestCommonPrefix (BVHSource/BVHAuxiliary.cuh:31-43).
 * ==================================================================================== */
static int clz32(uint32_t x) { return x ? __builtin_clz(x) : 32; }
static int clz64(uint64_t x) { return x ? __builtin_clzll(x) : 64; }
static int lcp_u32(const uint32_t* c, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  return c[i] != c[j] ? clz32(c[i] ^ c[j]) : clz32((uint32_t)(i ^ j)) + 32;
}
static int lcp_u64(const uint64_t* c, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  return c[i] != c[j] ? clz64(c[i] ^ c[j]) : clz32((uint32_t)(i ^ j)) + 64;
}
#define KARRAS_BODY(LCP)                                                                   \
  for (int i = 0; i < n - 1; ++i) {                                                        \
    int d = (LCP(codes, n, i, i + 1) - LCP(codes, n, i, i - 1)) > 0 ? 1 : -1;              \
    int sig_min = LCP(codes, n, i, i - d);                                                 \
    int lmax = 2;                                                                          \
    while (LCP(codes, n, i, i + lmax * d) > sig_min) lmax *= 2;                            \
    int l = 0, t;                                                                          \
    for (t = lmax / 2; t >= 1; t /= 2) {                                                   \
      if (LCP(codes, n, i, i + (l + t) * d) > sig_min) l += t;                             \
      if (t == 1) break;                                                                   \
    }                                                                                      \
    int j = i + l * d;                                                                     \
    int sig_node = LCP(codes, n, i, j);                                                    \
    int s = 0;                                                                             \
    double div;                                                                            \
    for (div = 2; t >= 1; div *= 2) {                                                      \
      t = (int)ceil((double)l / div);                                                      \
      if (LCP(codes, n, i, i + (s + t) * d) > sig_node) s += t;                            \
      if (t == 1) break;                                                                   \
    }                                                                                      \
    int gamma = i + s * d + (d < 0 ? d : 0);                                               \
    int node = n + i;                                                                      \
    int lo = i < j ? i : j, hi = i < j ? j : i;                                            \
    is_leaf[node] = 0;                                                                     \
    int lc = (lo == gamma) ? gamma : gamma + n;                                            \
    int rc = (hi == gamma + 1) ? gamma + 1 : gamma + 1 + n;                                \
    left[node] = lc; right[node] = rc;                                                     \
    parent[lc] = node; parent[rc] = node;                                                  \
    min_r[node] = lo; max_r[node] = hi;                                                    \
  }
void or_radix_tree_u32(const uint32_t* codes, int n, uint8_t* is_leaf, int* left, int* right,
                       int* parent, int* min_r, int* max_r) {
  KARRAS_BODY(lcp_u32)
}
void or_radix_tree_u64(const uint64_t* codes, int n, uint8_t* is_leaf, int* left, int* right,
                       int* parent, int* min_r, int* max_r) {
  KARRAS_BODY(lcp_u64)
}

/* (a10) leaves -- kernelConstructLeafNodesSoA (BVHSoAKernels.cu:108-138), initBound
 * (BVHAuxiliary.cuh:53-68).  bounds: 8 floats per node. */
void or_leaves(int n, const int* sorted_idx, const float* pos4, float r, uint8_t* is_leaf,
               int* min_r, int* max_r, float* cms4, float* bounds8) {
  for (int i = 0; i < n; ++i) {
    const float* c = pos4 + 4l * sorted_idx[i];
    is_leaf[i] = 1;
    min_r[i] = max_r[i] = i;
    memcpy(cms4 + 4l * i, c, 16);
    float* b = bounds8 + 8l * i;
    b[0] = c[0] - r; b[1] = c[1] - r; b[2] = c[2] - r;
    b[3] = c[0] + r; b[4] = c[1] + r; b[5] = c[2] + r;
    b[6] = 0.f; b[7] = 0.f;
  }
}

/* (a11) refit -- kernelConstructInternalNodesSoA (BVHSoAKernels.cu:148-176), mergeBounds
 * (BVHAuxiliary.cuh:83-94); done as a post-order walk from the root. */
static void refit_rec(int node, int n, const int* left, const int* right, float* b) {
  if (node < n) return;
  int a = left[node], c = right[node];
  refit_rec(a, n, left, right, b);
  refit_rec(c, n, left, right, b);
  float* A = b + 8l * a; float* C = b + 8l * c; float* R = b + 8l * node;
  for (int k = 0; k < 3; ++k) R[k] = A[k] < C[k] ? A[k] : C[k];
  for (int k = 3; k < 6; ++k) R[k] = A[k] > C[k] ? A[k] : C[k];
  R[6] = 0.f; R[7] = 0.f;
}
void or_refit(int n, const int* left, const int* right, float* bounds8) {
  if (n >= 2) refit_rec(n, n, left, right, bounds8);
}

/* ====================================================================================
 * (a12) BVH traversal with the reference's explicit stack -- collideBVHSoARigidBody
 * (Kernels/RB_BVHKernels.cu:100-244) with collideStaticSpheresBVH (:24-98) and checkOverlap
 * (BVHSource/BVHAuxiliary.cuh:139-152).  prm: r-independent DEM constants
 * {spring, damping, shear, attraction}.
 * ==================================================================================== */
static int overlap8(const float* a, const float* b) {
  return (a[0] <= b[3] && a[3] >= b[0]) && (a[1] <= b[4] && a[4] >= b[1]) &&
         (a[2] <= b[5] && a[5] >= b[2]);
}
static v3 spring_force(v3 rp, float dist, v3 rv, float contact, const float* prm) {
  v3 nrm = divs(rp, dist);
  v3 tv = sub(rv, scl(dot(rv, nrm), nrm));
  v3 f = scl(-prm[0] * (contact - dist), nrm);
  f = add(f, scl(prm[1], rv));
  f = add(f, scl(prm[2], tv));
  f = add(f, scl(prm[3], rp));
  return f;
}

/* Impulse on a particle at velocity vel from a static scene point with normal nn,
 * FindAndHandleAugmentedRealityCollisionsUniformGridCell (RigidBodies/UniformGridDEM.cu:275-296):
 * along -nn, the scene at rest (rv = 0 - vel), rp = point - particle, dist = |rp| < contact
 * tested by the caller.  prm = {spring, damping, shear, attraction}. */
static v3 scene_force(v3 rp, float dist, v3 vel, v3 nn, float contact, const float* prm) {
  v3 nrm = mk3(-nn.x, -nn.y, -nn.z);
  v3 rv = mk3(0.f - vel.x, 0.f - vel.y, 0.f - vel.z);
  v3 tv = sub(rv, scl(dot(rv, nrm), nrm));
  v3 f = scl(-prm[0] * (contact - dist), nrm);
  f = add(f, scl(prm[1], rv));
  f = add(f, scl(prm[2], tv));
  f = add(f, scl(prm[3], rp));
  return f;
}

static v3 static_pair(v4 pa, v4 pb, v4 cm, v3 va, v3 vb, float ra, float rb, const float* prm,
                      v4* corr) {
  v3 rp = mk3(pb.x - pa.x, pb.y - pa.y, pb.z - pa.z);
  float dist = sqrtf(dot(rp, rp));
  float cd = ra + rb;
  if (!(dist < cd)) return mk3(0.f, 0.f, 0.f);
  v3 f = spring_force(rp, dist, sub(vb, va), cd, prm);
  v3 nrm = divs(rp, dist);
  float offset = -(cd - dist) / 2.f;
  v3 cb = mk3(cm.x - pb.x, cm.y - pb.y, cm.z - pb.z);
  v3 ca = mk3(cm.x - pa.x, cm.y - pa.y, cm.z - pa.z);
  if (sqrtf(dot(cb, cb)) < sqrtf(dot(ca, ca))) offset = -offset;
  corr->x = nrm.x * offset; corr->y = nrm.y * offset; corr->z = nrm.z * offset; corr->w = 0.f;
  return f;
}
void or_collide_bvh_dem(const float* prm, const int* rb_idx, const float* rel4,
                        const float* vel4, const uint8_t* is_leaf, const int* left,
                        const int* right, const float* cms4, const float* bounds8,
                        const int* sorted_idx, const float* radii, int n, float* p_force4,
                        float* p_torque4, float* p_pos4) {
  if (n < 2) return;
#pragma omp parallel for schedule(dynamic, 256)
  for (int index = 0; index < n; ++index) {
    int local[256];
    int* st = local;
    int cap = 256;
    int* heap = NULL;
    int top = 0;
    int q = sorted_idx[index];
    v3 qvel = xyz(vel4 + 4l * q);
    v4 qpos = ld4(cms4 + 4l * index);
    float qrad = radii[index];
    int qbody = rb_idx[q];
    const float* qbox = bounds8 + 8l * index;
    v4 qr = ld4(rel4 + 4l * q);
    v4 rbcm = {qpos.x - qr.x, qpos.y - qr.y, qpos.z - qr.z, qpos.w - qr.w};
    v3 r3 = mk3(qr.x, qr.y, qr.z);
    v3 force = mk3(0.f, 0.f, 0.f), torque = mk3(0.f, 0.f, 0.f);
    v4 corr = {0.f, 0.f, 0.f, 0.f};
    st[top++] = -1;
    int node = n;
    do {
      int lc = left[node], rc = right[node];
      int ol = overlap8(qbox, bounds8 + 8l * lc), orr = overlap8(qbox, bounds8 + 8l * rc);
      if (lc == index) ol = 0;
      if (rc == index) orr = 0;
      int ll = is_leaf[lc], rl = is_leaf[rc];
      for (int side = 0; side < 2; ++side) {
        int c = side == 0 ? lc : rc;
        if (!((side == 0 ? ol : orr) && (side == 0 ? ll : rl))) continue;
        int oc = sorted_idx[c];
        if (!(qbody != rb_idx[oc] || qbody == -1)) continue;
        v4 lcorr = {0.f, 0.f, 0.f, 0.f};
        v3 f = static_pair(qpos, ld4(cms4 + 4l * c), rbcm, qvel, xyz(vel4 + 4l * oc), qrad,
                           radii[c], prm, &lcorr);
        if (side == 1) {
          corr.x = corr.x > lcorr.x ? corr.x : lcorr.x;
          corr.y = corr.y > lcorr.y ? corr.y : lcorr.y;
          corr.z = corr.z > lcorr.z ? corr.z : lcorr.z;
          corr.w = corr.w > lcorr.w ? corr.w : lcorr.w;
        }
        corr.x = corr.x + lcorr.x; corr.y = corr.y + lcorr.y;
        corr.z = corr.z + lcorr.z; corr.w = corr.w + lcorr.w;
        force = add(force, f);
        torque = add(torque, cross(r3, f));
      }
      int tl = ol && !ll, tr = orr && !rl;
      if (!tl && !tr) {
        node = st[--top];
      } else {
        node = tl ? lc : rc;
        if (tl && tr) {
          if (top == cap) {
            int* nh = (int*)malloc(sizeof(int) * cap * 2);
            memcpy(nh, st, sizeof(int) * cap);
            free(heap);
            heap = nh; st = nh; cap *= 2;
          }
          st[top++] = rc;
        }
      }
    } while (node != -1);
    free(heap);
    if (qbody == -1) continue;
    st4(p_force4 + 4l * q, force.x, force.y, force.z, 0.f);
    st4(p_torque4 + 4l * q, torque.x, torque.y, torque.z, 0.f);
    if (p_pos4) st4(p_pos4 + 4l * q, corr.x, corr.y, corr.z, corr.w);
  }
}

/* FindRigidBodyCollisionsBVHKernel (Kernels/RB_BVHKernels.cu:760-876), explicit stack. */
void or_find_contacts_bvh(const int* rb_idx, const uint8_t* is_leaf, const int* left,
                          const int* right, const int* max_r, const float* cms4,
                          const float* bounds8, const int* sorted_idx, const float* radii, int n,
                          float* contact_distance, int* colliding_particle,
                          int* colliding_body) {
  if (n < 2) return;
#pragma omp parallel for schedule(dynamic, 256)
  for (int index = 0; index < n; ++index) {
    int cap = 256, top = 0;
    int* st = (int*)malloc(sizeof(int) * cap);
    int q = sorted_idx[index];
    const float* qp = cms4 + 4l * index;
    const float* qbox = bounds8 + 8l * index;
    float qrad = radii[q];
    int qbody = rb_idx[q];
    float best = contact_distance[q];
    st[top++] = -1;
    int node = n;
    do {
      int lc = left[node], rc = right[node];
      int ol = overlap8(qbox, bounds8 + 8l * lc), orr = overlap8(qbox, bounds8 + 8l * rc);
      if (lc == index || max_r[lc] < index) ol = 0;
      if (rc == index || max_r[rc] < index) orr = 0;
      int ll = is_leaf[lc], rl = is_leaf[rc];
      for (int side = 0; side < 2; ++side) {
        int c = side == 0 ? lc : rc;
        if (!((side == 0 ? ol : orr) && (side == 0 ? ll : rl))) continue;
        int oc = sorted_idx[c], ob = rb_idx[oc];
        if (qbody == ob) continue;
        const float* cp = cms4 + 4l * c;
        float dx = cp[0] - qp[0], dy = cp[1] - qp[1], dz = cp[2] - qp[2], dw = cp[3] - qp[3];
        float dist = sqrtf(dx * dx + dy * dy + dz * dz + dw * dw);
        float thr = qrad + radii[oc];
        if (thr - dist > best) {
          best = thr - dist;
          contact_distance[q] = best;
          colliding_particle[q] = oc;
          colliding_body[q] = ob;
        }
      }
      int tl = ol && !ll, tr = orr && !rl;
      if (!tl && !tr) {
        node = st[--top];
      } else {
        node = tl ? lc : rc;
        if (tl && tr) {
          if (top == cap) { cap *= 2; st = (int*)realloc(st, sizeof(int) * cap); }
          st[top++] = rc;
        }
      }
    } while (node != -1);
    free(st);
  }
}

/* Contact pairs by brute force over all pairs (independent of any broad phase):
 * {i < j : |p_i - p_j| < two_r, body_i != body_j}, |v| = sqrtf(dot(v, v)) as in
 * RigidBodies/UniformGridDEM.cu:96-98.  Pairs written in (i, j) lexicographic order. */
long or_pairs_brute(const float* pos4, const int* rb_idx, int n, float two_r, int* pairs2,
                    long capacity) {
  long cnt = 0;
  for (int i = 0; i < n; ++i) {
    v3 pi = xyz(pos4 + 4l * i);
    for (int j = i + 1; j < n; ++j) {
      if (rb_idx[i] == rb_idx[j]) continue;
      v3 rp = sub(xyz(pos4 + 4l * j), pi);
      if (!(sqrtf(dot(rp, rp)) < two_r)) continue;
      if (cnt < capacity) { pairs2[2 * cnt] = i; pairs2[2 * cnt + 1] = j; }
      ++cnt;
    }
  }
  return cnt;
}

/* ====================================================================================
 * (a13) grid hash -- calcGridPos/calcGridHash/calcHashD (Kernels/particleKernels.cu:150-189).
 * grid: {ox, oy, oz, cx, cy, cz} floats, dims {gx, gy, gz} (powers of two).
 * ==================================================================================== */
typedef struct { float o[3], c[3]; uint32_t g[3]; } grid_t;
static void cell_of(const grid_t* G, v3 p, int* c) {
  c[0] = (int)floorf((p.x - G->o[0]) / G->c[0]);
  c[1] = (int)floorf((p.y - G->o[1]) / G->c[1]);
  c[2] = (int)floorf((p.z - G->o[2]) / G->c[2]);
}
static uint32_t hash3(const grid_t* G, int x, int y, int z) {
  uint32_t ux = (uint32_t)x & (G->g[0] - 1), uy = (uint32_t)y & (G->g[1] - 1),
           uz = (uint32_t)z & (G->g[2] - 1);
  return uz * G->g[1] * G->g[0] + uy * G->g[0] + ux;
}
void or_calc_hash(const float* grid6, const uint32_t* dims3, const float* pos4, long n,
                  uint32_t* hash) {
  grid_t G;
  memcpy(G.o, grid6, 12); memcpy(G.c, grid6 + 3, 12); memcpy(G.g, dims3, 12);
  for (long i = 0; i < n; ++i) {
    int c[3];
    cell_of(&G, xyz(pos4 + 4 * i), c);
    hash[i] = hash3(&G, c[0], c[1], c[2]);
  }
}

/* (a14) reorderDataAndFindCellStart (Kernels/particleKernels.cu:193-258 and the wrapper's
 * 0xffffffff memset, Kernels/particleKernelWrappers.cu:229) */
void or_reorder(const uint32_t* shash, const uint32_t* sidx, const float* pos4, const float* vel4,
                long n, long num_cells, uint32_t* cell_start, uint32_t* cell_end,
                float* spos4, float* svel4) {
  for (long c = 0; c < num_cells; ++c) cell_start[c] = EMPTY;
  for (long i = 0; i < n; ++i) {
    uint32_t h = shash[i];
    if (i == 0 || h != shash[i - 1]) {
      cell_start[h] = (uint32_t)i;
      if (i > 0) cell_end[shash[i - 1]] = (uint32_t)i;
    }
    if (i == n - 1) cell_end[h] = (uint32_t)(i + 1);
    memcpy(spos4 + 4 * i, pos4 + 4l * sidx[i], 16);
    if (svel4) memcpy(svel4 + 4 * i, vel4 + 4l * sidx[i], 16);
  }
}

/* (a15) FindAndHandleRigidBodyCollisionsUniformGridKernel (RigidBodies/UniformGridDEM.cu:
 * 57-204): per-cell partial sums, += into p_force / p_torque at the original index. */
void or_collide_grid_dem(const float* grid6, const uint32_t* dims3, const float* prm5,
                         const int* rb_idx, const float* spos4, const float* svel4,
                         const float* rel4, const uint32_t* gidx, const uint32_t* cstart,
                         const uint32_t* cend, long n, float* p_force4, float* p_torque4) {
  grid_t G;
  memcpy(G.o, grid6, 12); memcpy(G.c, grid6 + 3, 12); memcpy(G.g, dims3, 12);
  const float thr = 2.0f * prm5[4];
#pragma omp parallel for schedule(static)
  for (long index = 0; index < n; ++index) {
    v3 pos = xyz(spos4 + 4 * index), vel = xyz(svel4 + 4 * index);
    int gp[3];
    cell_of(&G, pos, gp);
    uint32_t orig = gidx[index];
    int body = rb_idx[orig];
    v3 lin = mk3(0.f, 0.f, 0.f);
    for (int z = -1; z <= 1; ++z)
      for (int y = -1; y <= 1; ++y)
        for (int x = -1; x <= 1; ++x) {
          v3 cf = mk3(0.f, 0.f, 0.f);
          uint32_t h = hash3(&G, gp[0] + x, gp[1] + y, gp[2] + z);
          uint32_t s = cstart[h];
          if (s != EMPTY) {
            uint32_t e = cend[h];
            for (uint32_t j = s; j < e; ++j) {
              int b2 = rb_idx[gidx[j]];
              if (j == (uint32_t)index || body == b2) continue;
              v3 rp = sub(xyz(spos4 + 4l * j), pos);
              float dist = sqrtf(dot(rp, rp));
              if (dist < thr) cf = add(cf, spring_force(rp, dist, sub(xyz(svel4 + 4l * j), vel), thr, prm5));
            }
          }
          lin = add(lin, cf);
        }
    float* F = p_force4 + 4l * orig;
    F[0] = F[0] + lin.x; F[1] = F[1] + lin.y; F[2] = F[2] + lin.z; F[3] = F[3] + 0.f;
    v3 t = cross(xyz(rel4 + 4l * orig), lin);
    float* T = p_torque4 + 4l * orig;
    T[0] = T[0] + t.x; T[1] = T[1] + t.y; T[2] = T[2] + t.z; T[3] = T[3] + 0.f;
  }
}

/* ====================================================================================
 * (a16) fixed-order per-body sum: lane l of a 32-lane warp adds elements s+l, s+l+32, ...,
 * then the lanes combine with a xor tree (16, 8, 4, 2, 1), lane l adding lane (l^o)'s value
 * to its own; the result is lane 0's.  (Replaces ReducePerParticleImpulses,
 * RigidBodies/UniformGridDEM.cu:462-666.)
 * ==================================================================================== */
static v3 warp_sum(const v3* vals, int count) {
  float x[32], y[32], z[32], nx[32], ny[32], nz[32];
  for (int l = 0; l < 32; ++l) { x[l] = 0.f; y[l] = 0.f; z[l] = 0.f; }
  for (int i = 0; i < count; ++i) {
    int l = i & 31;
    x[l] = x[l] + vals[i].x; y[l] = y[l] + vals[i].y; z[l] = z[l] + vals[i].z;
  }
  for (int o = 16; o > 0; o >>= 1) {
    for (int l = 0; l < 32; ++l) { nx[l] = x[l] + x[l ^ o]; ny[l] = y[l] + y[l ^ o]; nz[l] = z[l] + z[l ^ o]; }
    memcpy(x, nx, sizeof(x)); memcpy(y, ny, sizeof(y)); memcpy(z, nz, sizeof(z));
  }
  return mk3(x[0], y[0], z[0]);
}
void or_reduce_bodies(const float* pf4, const float* pt4, const int* off, int nb, float* bf4,
                      float* bt4) {
  for (int b = 0; b < nb; ++b) {
    int s = off[b], e = off[b + 1];
    v3* f = (v3*)malloc(sizeof(v3) * (e - s + 1));
    v3* t = (v3*)malloc(sizeof(v3) * (e - s + 1));
    for (int i = s; i < e; ++i) { f[i - s] = xyz(pf4 + 4l * i); t[i - s] = xyz(pt4 + 4l * i); }
    v3 F = warp_sum(f, e - s), T = warp_sum(t, e - s);
    st4(bf4 + 4l * b, F.x, F.y, F.z, 0.f);
    st4(bt4 + 4l * b, T.x, T.y, T.z, 0.f);
    free(f); free(t);
  }
}
/* CombineReducedImpulses (UniformGridDEM.cu:421-460) applied to the fixed-order sums. */
void or_reduce_impulses(const float* pf4, const float* pt4, const int* off, int nb, float* vel4,
                        float* ang4, const float* mass, const float* ib9) {
  float* bf = (float*)malloc(16l * (nb ? nb : 1));
  float* bt = (float*)malloc(16l * (nb ? nb : 1));
  or_reduce_bodies(pf4, pt4, off, nb, bf, bt);
  for (int b = 0; b < nb; ++b) {
    float m = mass[b];
    float* v = vel4 + 4l * b;
    v[0] = v[0] + bf[4 * b] / m; v[1] = v[1] + bf[4 * b + 1] / m;
    v[2] = v[2] + bf[4 * b + 2] / m; v[3] = v[3] + 0.f / m;
    v3 w = glm_mv(ib9 + 9l * b, xyz(bt + 4l * b));
    float* a = ang4 + 4l * b;
    a[0] = a[0] + w.x; a[1] = a[1] + w.y; a[2] = a[2] + w.z; a[3] = a[3] + 0.f;
  }
  free(bf); free(bt);
}

/* ====================================================================================
 * (a2) GPUintegratorKernel (Kernels/rigidBodyKernels.cu:262-348) and (a4)
 * computeGlobalAttributes + resetQuaternionKernel (:386-456), glm order of operations.
 * ==================================================================================== */
void or_integrate_reference(const float* gravity3, float w_damping, float dt, int nb,
                            float* cms4, float* vel4, float* ang4, float* quat4, const float* ib9,
                            float* cur9, float* model16, float* cum4) {
  for (int b = 0; b < nb; ++b) {
    float* p = cms4 + 4l * b;
    float* v = vel4 + 4l * b;
    v4 w4 = ld4(ang4 + 4l * b);
    st4(p, p[0] + v[0] * dt, p[1] + v[1] * dt, p[2] + v[2] * dt, p[3] + v[3] * dt);
    v3 nv = mk3(w4.x, w4.y, w4.z);
    float d = dot(nv, nv);
    float inv = 1.0f / sqrtf(d);
    v3 nrm = mk3(nv.x * inv, nv.y * inv, nv.z * inv);
    float theta = sqrtf(d) * dt;
    v4 q = {0.f, 0.f, 0.f, 1.f};
    if (theta > 0.00001f) {
      float c = cosf(theta / 2.f), s = sinf(theta / 2.f);
      q.x = s * nrm.x; q.y = s * nrm.y; q.z = s * nrm.z; q.w = c;
    }
    q = glm_qnormalize(q);
    float R[9], RI[9], Rt[9], C[9];
    glm_mat3_cast(q, R);
    glm_mm(R, ib9 + 9l * b, RI);
    for (int c = 0; c < 3; ++c) for (int r = 0; r < 3; ++r) Rt[c * 3 + r] = R[r * 3 + c];
    glm_mm(RI, Rt, C);
    memcpy(cur9 + 9l * b, C, 36);
    if (cum4) {
      v4 cq = glm_qnormalize(glm_qmul(q, ld4(cum4 + 4l * b)));
      st4(cum4 + 4l * b, cq.x, cq.y, cq.z, cq.w);
      if (model16) {
        float M[9];
        float* mo = model16 + 16l * b;
        glm_mat3_cast(cq, M);
        for (int c = 0; c < 3; ++c) {
          for (int r = 0; r < 3; ++r) mo[c * 4 + r] = M[c * 3 + r];
          mo[c * 4 + 3] = 0.f;
        }
        mo[12] = p[0]; mo[13] = p[1]; mo[14] = p[2]; mo[15] = 1.f;
      }
    }
    st4(v, v[0] + gravity3[0], v[1] + gravity3[1], v[2] + gravity3[2], v[3] + 0.f);
    st4(quat4 + 4l * b, q.x, q.y, q.z, q.w);
    st4(ang4 + 4l * b, nv.x * w_damping, nv.y * w_damping, nv.z * w_damping, 0.f * w_damping);
  }
}
void or_global_attributes(int n, int nb, const float* cms4, const float* rbvel4,
                          const float* rbang4, float* quat4, const int* rb_idx, float* rel4,
                          float* pos4, float* vel4) {
  for (int i = 0; i < n; ++i) {
    int b = rb_idx[i];
    if (b == -1) continue;
    float R[9];
    glm_mat3_cast(ld4(quat4 + 4l * b), R);
    float* r0 = rel4 + 4l * i;
    v3 r = mk3((R[0] * r0[0] + R[3] * r0[1]) + (R[6] * r0[2] + 0.f * 0.f),
               (R[1] * r0[0] + R[4] * r0[1]) + (R[7] * r0[2] + 0.f * 0.f),
               (R[2] * r0[0] + R[5] * r0[1]) + (R[8] * r0[2] + 0.f * 0.f));
    st4(r0, r.x, r.y, r.z, 0.f);
    const float* c = cms4 + 4l * b;
    st4(pos4 + 4l * i, r.x + c[0], r.y + c[1], r.z + c[2], 0.f + c[3]);
    const float* v = rbvel4 + 4l * b;
    v3 w = cross(xyz(rbang4 + 4l * b), r);
    st4(vel4 + 4l * i, v[0] + w.x, v[1] + w.y, v[2] + w.z, v[3] + 0.f);
  }
  for (int b = 0; b < nb; ++b) st4(quat4 + 4l * b, 0.f, 0.f, 0.f, 1.f);
}

/* ====================================================================================
 * (a18) WallCollisionWrapper (WallCollisions.cu:46-129, 201-276, 338-597): deepest admissible
 * wall per particle, deepest contact per body (ties -> larger particle index), Baraff e = 1.
 * ==================================================================================== */
static float dot4f(v4 a, v4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
void or_walls_reference(float radius, const float* ppos4, const float* rbpos4,
                        const float* mn3, const float* mx3, float* rbvel4, float* rbang4,
                        const float* ib9, const float* mass, const int* rb_idx, const int* off,
                        int nb) {
  float wpos[6] = {mx3[0], mx3[1], mx3[2], mn3[0], mn3[1], mn3[2]};
  /* detection uses the velocities before any impulse */
  float* vel0 = (float*)malloc(16l * (nb ? nb : 1));
  memcpy(vel0, rbvel4, 16l * nb);
  for (int b = 0; b < nb; ++b) {
    float best_d = 0.f;
    int best_i = -1, best_w = 0;
    for (int i = off[b]; i < off[b + 1]; ++i) {
      int body = rb_idx[i];
      if (body == -1) continue;
      v4 v = ld4(vel0 + 4l * body), p = ld4(ppos4 + 4l * i);
      float cd = 0.f;
      int cw = -1;
      for (int w = 0; w < 6; ++w) {
        float s = w < 3 ? 1.f : -1.f;
        int a = w % 3;
        v4 nrm = {a == 0 ? s : 0.f, a == 1 ? s : 0.f, a == 2 ? s : 0.f, 0.f};
        float sign = nrm.x * 1.f + nrm.y * 1.f + nrm.z * 1.f + nrm.w * 0.f;
        v4 nn = {nrm.x * sign, nrm.y * sign, nrm.z * sign, nrm.w * sign};
        float dist = sign * (dot4f(p, nn) - wpos[w] + radius * sign);
        if (dist > cd && dot4f(v, nrm) > 0.f) { cd = dist; cw = w; }
      }
      if (cw >= 0 && (best_i < 0 || cd >= best_d)) { best_d = cd; best_i = i; best_w = cw; }
    }
    if (best_i < 0 || !(best_d > 0.f)) continue;
    float s = best_w < 3 ? 1.f : -1.f;
    int a = best_w % 3;
    v4 n = {a == 0 ? s : 0.f, a == 1 ? s : 0.f, a == 2 ? s : 0.f, 0.f};
    float wp = wpos[best_w];
    v4 wall = {n.x * wp, n.y * wp, n.z * wp, n.w * wp};
    v4 p = ld4(ppos4 + 4l * best_i);
    float pd = dot4f(p, n);
    v4 paux = {n.x * pd, n.y * pd, n.z * pd, n.w * pd};
    v4 ocm = ld4(rbpos4 + 4l * b), ov = ld4(rbvel4 + 4l * b), oa = ld4(rbang4 + 4l * b);
    const float* I = ib9 + 9l * b;
    float m = mass[b];
    v4 disp = {p.x - ocm.x, p.y - ocm.y, p.z - ocm.z, p.w - ocm.w};
    v4 rn = {radius * n.x, radius * n.y, radius * n.z, radius * n.w};
    v4 ncm = {((ocm.x + wall.x) - rn.x) - paux.x, ((ocm.y + wall.y) - rn.y) - paux.y,
              ((ocm.z + wall.z) - rn.z) - paux.z, ((ocm.w + wall.w) - rn.w) - paux.w};
    v4 np = {ncm.x + disp.x, ncm.y + disp.y, ncm.z + disp.z, 1.f};
    v4 p2 = {np.x + n.x * radius, np.y + n.y * radius, np.z + n.z * radius, np.w + n.w * radius};
    float t = radius / (radius + 0.f);
    v4 dp = {p2.x - np.x, p2.y - np.y, p2.z - np.z, p2.w - np.w};
    v4 cp = {np.x + dp.x * t, np.y + dp.y * t, np.z + dp.z * t, np.w + dp.w * t};
    float il = 1.0f / sqrtf(dot4f(dp, dp));
    v4 cn = {dp.x * il * -1.f, dp.y * il * -1.f, dp.z * il * -1.f, dp.w * il * -1.f};
    v4 r = {ncm.x - cp.x, ncm.y - cp.y, ncm.z - cp.z, ncm.w - cp.w};
    v3 v3v = mk3(ov.x, ov.y, ov.z), w3 = mk3(oa.x, oa.y, oa.z);
    v3 r3 = mk3(r.x, r.y, r.z), n3 = mk3(cn.x, cn.y, cn.z);
    v3 va = add(v3v, glm_cross(w3, r3));
    float numer = -(1.f + 1.f) * dot(va, n3);
    float aa = 1.f / m;
    float bb = dot(glm_cross(glm_mv(I, glm_cross(r3, n3)), r3), n3);
    float j = numer / (aa + bb);
    v4 lin = {cn.x * j, cn.y * j, cn.z * j, cn.w * j};
    v3 ai = glm_mv(I, glm_cross(r3, mk3(lin.x, lin.y, lin.z)));
    st4(rbvel4 + 4l * b, ov.x + lin.x / m, ov.y + lin.y / m, ov.z + lin.z / m, ov.w + lin.w / m);
    st4(rbang4 + 4l * b, oa.x + ai.x, oa.y + ai.y, oa.z + ai.z, oa.w + 0.f);
  }
  free(vel0);
}

/* ====================================================================================
 * Fused PHYSICAL step (the product's ar_step), float32, operation for operation:
 *   re-pose + hash -> stable sort -> cell ranges -> DEM gather + walls (+ the static point
 *   cloud's impulses, or_step_ex) -> fixed-order body sums of F and r x F -> semi-implicit
 *   Euler.
 * scene12 = {bmin[3], bmax[3], g[3], r, dt, k}, scene3 = {damping, shear, attraction},
 * grid: origin[3], cell[3], dims[3].  rel4.w holds the body index (int bits).
 * Outputs (optional): sorted keys and indices, per-particle force, per-body sums.
 * ==================================================================================== */
typedef struct {
  float bmin[3], bmax[3], g[3], r, dt, k, damping, shear, attraction;
  grid_t G;
} scene_t;

static v3 wall_force(const scene_t* s, v3 p, v3 v) {
  v3 f = mk3(0.f, 0.f, 0.f);
  float pc[3] = {p.x, p.y, p.z};
  v3 rv = mk3(-v.x, -v.y, -v.z);
  for (int a = 0; a < 3; ++a)
    for (int side = 0; side < 2; ++side) {
      float d = side == 0 ? pc[a] - s->bmin[a] : s->bmax[a] - pc[a];
      if (!(d < s->r)) continue;
      float sgn = side == 0 ? 1.f : -1.f;
      v3 tv = rv;
      if (a == 0) tv.x = 0.f; else if (a == 1) tv.y = 0.f; else tv.z = 0.f;
      v3 fw = add(scl(s->damping, rv), scl(s->shear, tv));
      float push = sgn * (s->k * (s->r - d));
      if (a == 0) fw.x = fw.x + push; else if (a == 1) fw.y = fw.y + push; else fw.z = fw.z + push;
      f = add(f, fw);
    }
  return f;
}

static int integrate_body(const scene_t* s, v3 F, v3 T, float m, const float* ib, float* pos,
                          float* quat, float* vel, float* ang) {
  float dt = s->dt;
  v4 q = ld4(quat);
  v3 acc = add(mk3(s->g[0], s->g[1], s->g[2]), divs(F, m));
  v3 nv = add(xyz(vel), scl(dt, acc));
  v4 qc = {-q.x, -q.y, -q.z, q.w};
  v3 tb = quat_rotate(qc, T);
  v3 lb = glm_mv(ib, tb);
  v3 dw = quat_rotate(q, lb);
  v3 nw = add(xyz(ang), scl(dt, dw));
  v3 nc = add(xyz(pos), scl(dt, nv));
  v4 wq = {nw.x, nw.y, nw.z, 0.f};
  v4 qd = glm_qmul(wq, q);
  float h = 0.5f * dt;
  v4 nq = {q.x + h * qd.x, q.y + h * qd.y, q.z + h * qd.z, q.w + h * qd.w};
  float inv = 1.f / sqrtf(((nq.x * nq.x + nq.y * nq.y) + nq.z * nq.z) + nq.w * nq.w);
  nq.x = nq.x * inv; nq.y = nq.y * inv; nq.z = nq.z * inv; nq.w = nq.w * inv;
  pos[0] = nc.x; pos[1] = nc.y; pos[2] = nc.z;
  vel[0] = nv.x; vel[1] = nv.y; vel[2] = nv.z;
  ang[0] = nw.x; ang[1] = nw.y; ang[2] = nw.z;
  quat[0] = nq.x; quat[1] = nq.y; quat[2] = nq.z; quat[3] = nq.w;
  float chk = nc.x + nc.y + nc.z + nv.x + nv.y + nv.z + nw.x + nw.y + nw.z + nq.x + nq.y + nq.z + nq.w;
  return isfinite(chk);
}

static void scene_from(const float* s15, const float* grid6, const uint32_t* dims3, scene_t* s) {
  memcpy(s->bmin, s15, 12); memcpy(s->bmax, s15 + 3, 12); memcpy(s->g, s15 + 6, 12);
  s->r = s15[9]; s->dt = s15[10]; s->k = s15[11];
  s->damping = s15[12]; s->shear = s15[13]; s->attraction = s15[14];
  memcpy(s->G.o, grid6, 12); memcpy(s->G.c, grid6 + 3, 12); memcpy(s->G.g, dims3, 12);
}

static long lower_bound_u32(const uint32_t* a, long n, uint32_t v) {
  long lo = 0, hi = n;
  while (lo < hi) { long mid = (lo + hi) / 2; if (a[mid] < v) lo = mid + 1; else hi = mid; }
  return lo;
}

/* Per body: fixed-order sums of F and r x F (warp_sum), then integrate_body.  0 on a
 * non-finite state. */
static int bodies_step(const scene_t* S, int nb, const float* pf, float* bpos4, float* bquat4,
                       float* bvel4, float* bang4, const float* mass, const float* ib9,
                       const int* off, const float* rel4, float* bforce4_out,
                       float* btorque4_out) {
  int ok = 1;
  for (int b = 0; b < nb; ++b) {
    int s0 = off[b], s1 = off[b + 1];
    v3* fv = (v3*)malloc(sizeof(v3) * (s1 - s0 + 1));
    v3* tv = (v3*)malloc(sizeof(v3) * (s1 - s0 + 1));
    v4 q = ld4(bquat4 + 4l * b);
    for (int i = s0; i < s1; ++i) {
      v3 f = xyz(pf + 4l * i);
      fv[i - s0] = f;
      tv[i - s0] = cross(quat_rotate(q, xyz(rel4 + 4l * i)), f);
    }
    v3 F = warp_sum(fv, s1 - s0), T = warp_sum(tv, s1 - s0);
    free(fv); free(tv);
    if (!integrate_body(S, F, T, mass[b], ib9 + 9l * b, bpos4 + 4l * b, bquat4 + 4l * b,
                        bvel4 + 4l * b, bang4 + 4l * b))
      ok = 0;
    if (bforce4_out) st4(bforce4_out + 4l * b, F.x, F.y, F.z, 0.f);
    if (btorque4_out) st4(btorque4_out + 4l * b, T.x, T.y, T.z, 0.f);
  }
  return ok;
}

/* or_step with a static point cloud of cm points (cloud_pos4, cloud_norm4; cm = 0: none): the
 * cloud is sorted by (cell key, index) in the same grid once; after a particle's contacts and
 * walls, the cloud points in its 27 neighbour cells (z, y, x order, a cell's points in sorted
 * order, per-cell partial sums) with |rp| < 2r add scene_force, and the cloud total is added
 * to the particle's force (the simulateAR branch of updateUniformGridDEM,
 * RigidBodies/UniformGridUpdate.cpp:967-969, with the kernel of
 * RigidBodies/UniformGridDEM.cu:301-377). */
int or_step_ex(const float* s15, const float* grid6, const uint32_t* dims3, int nb, int n,
               float* bpos4, float* bquat4, float* bvel4, float* bang4, const float* mass,
               const float* ib9, const int* off, const float* rel4, int steps,
               uint32_t* skeys_out, uint32_t* sidx_out, float* pforce4_out, float* bforce4_out,
               float* btorque4_out, const float* cloud_pos4, const float* cloud_norm4, int cm) {
  scene_t S;
  scene_from(s15, grid6, dims3, &S);
  const int key_bits = 32;
  uint32_t* ck = NULL;  /* the cloud's sorted keys and points, normals in the same order */
  float *cp = NULL, *cn = NULL;
  if (cm > 0) {
    uint32_t* k0 = (uint32_t*)malloc(4l * cm);
    uint32_t* ci = (uint32_t*)malloc(4l * cm);
    ck = (uint32_t*)malloc(4l * cm);
    cp = (float*)malloc(16l * cm);
    cn = (float*)malloc(16l * cm);
    for (int i = 0; i < cm; ++i) {
      int c[3];
      cell_of(&S.G, xyz(cloud_pos4 + 4l * i), c);
      k0[i] = hash3(&S.G, c[0], c[1], c[2]);
    }
    or_sort_pairs_u32(k0, NULL, ck, ci, cm, 0, key_bits);
    for (int j = 0; j < cm; ++j) {
      memcpy(cp + 4l * j, cloud_pos4 + 4l * ci[j], 16);
      memcpy(cn + 4l * j, cloud_norm4 + 4l * ci[j], 16);
    }
    free(k0); free(ci);
  }
  uint32_t* keys = (uint32_t*)malloc(4l * n);
  uint32_t* sk = (uint32_t*)malloc(4l * n);
  uint32_t* sv = (uint32_t*)malloc(4l * n);
  float* sp = (float*)malloc(16l * n);
  float* svl = (float*)malloc(16l * n);
  float* pf = (float*)malloc(16l * n);
  int ok = 1;
  for (int step = 0; step < steps; ++step) {
    for (int i = 0; i < n; ++i) {
      int b = f2i(rel4[4l * i + 3]);
      v3 r = quat_rotate(ld4(bquat4 + 4l * b), xyz(rel4 + 4l * i));
      v3 p = add(xyz(bpos4 + 4l * b), r);
      int c[3];
      cell_of(&S.G, p, c);
      keys[i] = hash3(&S.G, c[0], c[1], c[2]);
    }
    or_sort_pairs_u32(keys, NULL, sk, sv, n, 0, key_bits);
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n; ++k) {
      int g = (int)sv[k];
      int b = f2i(rel4[4l * g + 3]);
      v4 q = ld4(bquat4 + 4l * b);
      v3 r = quat_rotate(q, xyz(rel4 + 4l * g));
      v3 p = add(xyz(bpos4 + 4l * b), r);
      v3 v = add(xyz(bvel4 + 4l * b), cross(xyz(bang4 + 4l * b), r));
      st4(sp + 4l * k, p.x, p.y, p.z, i2f(b));
      st4(svl + 4l * k, v.x, v.y, v.z, 0.f);
    }
    const float thr = 2.0f * S.r;
    const float prm[4] = {S.k, S.damping, S.shear, S.attraction};
#pragma omp parallel for schedule(static)
    for (int k = 0; k < n; ++k) {
      v3 pos = xyz(sp + 4l * k), vel = xyz(svl + 4l * k);
      int body = f2i(sp[4l * k + 3]);
      int gp[3];
      cell_of(&S.G, pos, gp);
      v3 lin = mk3(0.f, 0.f, 0.f);
      for (int z = -1; z <= 1; ++z)
        for (int y = -1; y <= 1; ++y)
          for (int x = -1; x <= 1; ++x) {
            v3 cf = mk3(0.f, 0.f, 0.f);
            uint32_t h = hash3(&S.G, gp[0] + x, gp[1] + y, gp[2] + z);
            long s = lower_bound_u32(sk, n, h);
            for (long j = s; j < n && sk[j] == h; ++j) {
              if (j == k || f2i(sp[4l * j + 3]) == body) continue;
              v3 rp = sub(xyz(sp + 4l * j), pos);
              float dist = sqrtf(dot(rp, rp));
              if (dist < thr) cf = add(cf, spring_force(rp, dist, sub(xyz(svl + 4l * j), vel), thr, prm));
            }
            lin = add(lin, cf);
          }
      lin = add(lin, wall_force(&S, pos, vel));
      if (cm > 0) {
        v3 tot = mk3(0.f, 0.f, 0.f);
        for (int z = -1; z <= 1; ++z)
          for (int y = -1; y <= 1; ++y)
            for (int x = -1; x <= 1; ++x) {
              v3 cf = mk3(0.f, 0.f, 0.f);
              uint32_t h = hash3(&S.G, gp[0] + x, gp[1] + y, gp[2] + z);
              for (long j = lower_bound_u32(ck, cm, h); j < cm && ck[j] == h; ++j) {
                v3 rp = sub(xyz(cp + 4l * j), pos);
                float dist = sqrtf(dot(rp, rp));
                if (dist < thr) cf = add(cf, scene_force(rp, dist, vel, xyz(cn + 4l * j), thr, prm));
              }
              tot = add(tot, cf);
            }
        lin = add(lin, tot);
      }
      st4(pf + 4l * sv[k], lin.x, lin.y, lin.z, 0.f);
    }
    if (!bodies_step(&S, nb, pf, bpos4, bquat4, bvel4, bang4, mass, ib9, off, rel4, bforce4_out,
                     btorque4_out))
      ok = 0;
  }
  if (skeys_out) memcpy(skeys_out, sk, 4l * n);
  if (sidx_out) memcpy(sidx_out, sv, 4l * n);
  if (pforce4_out) memcpy(pforce4_out, pf, 16l * n);
  free(keys); free(sk); free(sv); free(sp); free(svl); free(pf);
  free(ck); free(cp); free(cn);
  return ok;
}

int or_step(const float* s15, const float* grid6, const uint32_t* dims3, int nb, int n,
            float* bpos4, float* bquat4, float* bvel4, float* bang4, const float* mass,
            const float* ib9, const int* off, const float* rel4, int steps, uint32_t* skeys_out,
            uint32_t* sidx_out, float* pforce4_out, float* bforce4_out, float* btorque4_out) {
  return or_step_ex(s15, grid6, dims3, nb, n, bpos4, bquat4, bvel4, bang4, mass, ib9, off, rel4,
                    steps, skeys_out, sidx_out, pforce4_out, bforce4_out, btorque4_out, NULL,
                    NULL, 0);
}

/* ====================================================================================
 * Fused PHYSICAL step with the BVH broad phase (the product's ar_step on a BVH scene):
 *   30-bit Morton code of each particle's world position normalised to the scene box
 *   (morton3D / expandBits, BVHSource/BVHkernels.cu:646-716) -> stable sort -> Karras tree
 *   with the index tie-break (or_radix_tree_u64) -> leaf boxes p +/- r -> refit -> per particle
 *   the explicit-stack traversal of collideBVHSoARigidBody (Kernels/RB_BVHKernels.cu:100-244),
 *   contacts summed in visit order, then the walls -> the same body sums and integration as
 *   or_step.  s15 as in or_step.  Outputs (optional): sorted codes and indices, per-particle
 *   force, per-body sums.
 * ==================================================================================== */
static uint32_t morton_box(v3 p, const float* lo, const float* hi) {
  uint32_t q[3];
  q[0] = quantise((p.x - lo[0]) / (hi[0] - lo[0]), 1024.0f, 1023.0f);
  q[1] = quantise((p.y - lo[1]) / (hi[1] - lo[1]), 1024.0f, 1023.0f);
  q[2] = quantise((p.z - lo[2]) / (hi[2] - lo[2]), 1024.0f, 1023.0f);
  uint32_t c = 0;
  for (int b = 0; b < 10; ++b)
    c |= (((q[0] >> b) & 1u) << (3 * b + 2)) | (((q[1] >> b) & 1u) << (3 * b + 1)) |
         (((q[2] >> b) & 1u) << (3 * b));
  return c;
}
int or_step_bvh(const float* s15, int nb, int n, float* bpos4, float* bquat4, float* bvel4,
                float* bang4, const float* mass, const float* ib9, const int* off,
                const float* rel4, int steps, uint64_t* skeys_out, uint32_t* sidx_out,
                float* pforce4_out, float* bforce4_out, float* btorque4_out) {
  scene_t S;
  const float g6[6] = {0, 0, 0, 1, 1, 1};
  const uint32_t d3[3] = {1, 1, 1};
  scene_from(s15, g6, d3, &S);
  uint64_t* keys = (uint64_t*)malloc(8l * n + 8);
  uint64_t* sk = (uint64_t*)malloc(8l * n + 8);
  uint32_t* sv = (uint32_t*)malloc(4l * n + 4);
  float* sp = (float*)malloc(16l * n + 16);
  float* svl = (float*)malloc(16l * n + 16);
  float* pf = (float*)malloc(16l * n + 16);
  const long m = 2l * n + 2;
  uint8_t* is_leaf = (uint8_t*)calloc(m, 1);
  int* left = (int*)calloc(m, sizeof(int));
  int* right = (int*)calloc(m, sizeof(int));
  int* parent = (int*)calloc(m, sizeof(int));
  int* min_r = (int*)calloc(m, sizeof(int));
  int* max_r = (int*)calloc(m, sizeof(int));
  float* bounds = (float*)calloc(8 * m, sizeof(float));
  int ok = 1;
  for (int step = 0; step < steps; ++step) {
    for (int i = 0; i < n; ++i) {
      int b = f2i(rel4[4l * i + 3]);
      v3 r = quat_rotate(ld4(bquat4 + 4l * b), xyz(rel4 + 4l * i));
      v3 p = add(xyz(bpos4 + 4l * b), r);
      keys[i] = morton_box(p, S.bmin, S.bmax);
    }
    or_sort_pairs_u64(keys, NULL, sk, sv, n, 0, 30);
    for (int k = 0; k < n; ++k) {
      int g = (int)sv[k];
      int b = f2i(rel4[4l * g + 3]);
      v4 q = ld4(bquat4 + 4l * b);
      v3 r = quat_rotate(q, xyz(rel4 + 4l * g));
      v3 p = add(xyz(bpos4 + 4l * b), r);
      v3 v = add(xyz(bvel4 + 4l * b), cross(xyz(bang4 + 4l * b), r));
      st4(sp + 4l * k, p.x, p.y, p.z, i2f(b));
      st4(svl + 4l * k, v.x, v.y, v.z, 0.f);
      float* bb = bounds + 8l * k;
      bb[0] = p.x - S.r; bb[1] = p.y - S.r; bb[2] = p.z - S.r;
      bb[3] = p.x + S.r; bb[4] = p.y + S.r; bb[5] = p.z + S.r;
      bb[6] = 0.f; bb[7] = 0.f;
      is_leaf[k] = 1;
      min_r[k] = max_r[k] = k;
    }
    if (n >= 2) {
      or_radix_tree_u64(sk, n, is_leaf, left, right, parent, min_r, max_r);
      or_refit(n, left, right, bounds);
    }
    const float thr = 2.0f * S.r;
    const float prm[4] = {S.k, S.damping, S.shear, S.attraction};
#pragma omp parallel for schedule(dynamic, 256)
    for (int k = 0; k < n; ++k) {
      v3 pos = xyz(sp + 4l * k), vel = xyz(svl + 4l * k);
      int body = f2i(sp[4l * k + 3]);
      const float* qbox = bounds + 8l * k;
      v3 lin = mk3(0.f, 0.f, 0.f);
      if (n >= 2) {
        int cap = 64, top = 0;
        int* st = (int*)malloc(sizeof(int) * cap);
        st[top++] = -1;
        int node = n;
        do {
          int lc = left[node], rc = right[node];
          int ol = lc != k && overlap8(qbox, bounds + 8l * lc);
          int orr = rc != k && overlap8(qbox, bounds + 8l * rc);
          int ll = is_leaf[lc], rl = is_leaf[rc];
          for (int side = 0; side < 2; ++side) {
            int c = side == 0 ? lc : rc;
            if (!((side == 0 ? ol : orr) && (side == 0 ? ll : rl))) continue;
            if (f2i(sp[4l * c + 3]) == body) continue;
            v3 rp = sub(xyz(sp + 4l * c), pos);
            float dist = sqrtf(dot(rp, rp));
            if (dist < thr) lin = add(lin, spring_force(rp, dist, sub(xyz(svl + 4l * c), vel), thr, prm));
          }
          int tl = ol && !ll, tr = orr && !rl;
          if (!tl && !tr) {
            node = st[--top];
          } else {
            node = tl ? lc : rc;
            if (tl && tr) {
              if (top == cap) { cap *= 2; st = (int*)realloc(st, sizeof(int) * cap); }
              st[top++] = rc;
            }
          }
        } while (node != -1);
        free(st);
      }
      lin = add(lin, wall_force(&S, pos, vel));
      st4(pf + 4l * sv[k], lin.x, lin.y, lin.z, 0.f);
    }
    if (!bodies_step(&S, nb, pf, bpos4, bquat4, bvel4, bang4, mass, ib9, off, rel4, bforce4_out,
                     btorque4_out))
      ok = 0;
  }
  if (skeys_out) memcpy(skeys_out, sk, 8l * n);
  if (sidx_out) memcpy(sidx_out, sv, 4l * n);
  if (pforce4_out) memcpy(pforce4_out, pf, 16l * n);
  free(keys); free(sk); free(sv); free(sp); free(svl); free(pf);
  free(is_leaf); free(left); free(right); free(parent); free(min_r); free(max_r); free(bounds);
  return ok;
}

/* ====================================================================================
 * AR static scene against the particles -- FindAndHandleAugmentedRealityCollisionsUniform-
 * GridCell / Kernel (RigidBodies/UniformGridDEM.cu:243-377).  The scene's particles are
 * sorted into the same grid with their own cell table; normals are unsorted.
 * prm = {spring, damping, shear, attraction}.  lin4 / ang4 are accumulated in place; color4
 * (may be NULL) is set to (0, 1, 0, 0) for particles with a contact.
 * ==================================================================================== */
void or_collide_static_scene(const float* grid6, const uint32_t* dims3, float radius,
                             const float* prm, const float* spos4, const float* svel4,
                             const float* rel4, const float* scene_spos4,
                             const float* scene_normals4, const uint32_t* gidx,
                             const uint32_t* scene_gidx, const uint32_t* cstart,
                             const uint32_t* cend, int n, float* lin4, float* ang4,
                             float* color4) {
  grid_t G;
  memcpy(G.o, grid6, 12); memcpy(G.c, grid6 + 3, 12); memcpy(G.g, dims3, 12);
  const float thr = 2.0f * radius;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < n; ++k) {
    v3 pos = xyz(spos4 + 4l * k), vel = xyz(svel4 + 4l * k);
    int gp[3];
    cell_of(&G, pos, gp);
    uint32_t orig = gidx[k];
    int contacts = 0;
    float lin[4] = {0.f, 0.f, 0.f, 0.f};
    for (int z = -1; z <= 1; ++z)
      for (int y = -1; y <= 1; ++y)
        for (int x = -1; x <= 1; ++x) {
          float cf[4] = {0.f, 0.f, 0.f, 0.f};
          uint32_t h = hash3(&G, gp[0] + x, gp[1] + y, gp[2] + z);
          if (cstart[h] != 0xffffffffu) {
            for (uint32_t j = cstart[h]; j < cend[h]; ++j) {
              uint32_t o2 = scene_gidx[j];
              v3 rp = sub(xyz(scene_spos4 + 4l * j), pos);
              float dist = sqrtf(dot(rp, rp));
              if (!(dist < thr)) continue;
              v3 f = scene_force(rp, dist, vel, xyz(scene_normals4 + 4l * o2), thr, prm);
              cf[0] = cf[0] + f.x; cf[1] = cf[1] + f.y; cf[2] = cf[2] + f.z; cf[3] = cf[3] + 0.f;
              ++contacts;
            }
          }
          for (int c = 0; c < 4; ++c) lin[c] = lin[c] + cf[c];
        }
    if (contacts && color4) st4(color4 + 4l * orig, 0.f, 1.f, 0.f, 0.f);
    float* L = lin4 + 4l * orig;
    st4(L, L[0] + lin[0], L[1] + lin[1], L[2] + lin[2], L[3] + lin[3]);
    v3 t = cross(xyz(rel4 + 4l * orig), mk3(lin[0], lin[1], lin[2]));
    float* A = ang4 + 4l * orig;
    st4(A, A[0] + t.x, A[1] + t.y, A[2] + t.z, A[3] + 0.f);
  }
}

/* ====================================================================================
 * AR static scene, impulse variant -- ARcollisionsUniformGridKernel / ARCellRigidBody /
 * collideARSpheresBaraffExact (Kernels/RB_UniformGridKernels.cu:420-678).  Each of the 27
 * iterations of the neighbour loop examines the particle's own cell (the reference passes
 * gridPos, :613).  Impulse j = -(1 + e)(v . n) / (((I^-1 (r x n)) x r) . n + 1/m) along
 * n = (p - q) / |p - q|, r = contact point - (p - rel).  inertia9: glm::mat3 per body.
 * Particles of a body: force, torque, count at the original index; free particles (body -1):
 * force added to new_vel4, with a zero inverse inertia and unit mass.
 * ==================================================================================== */
void or_ar_collide_impulse(const float* grid6, const uint32_t* dims3, float radius,
                           float restitution, const int* rb_idx, const float* rel4,
                           const float* inertia9, const float* mass, const float* scene_radii,
                           const float* spos4, const float* svel4, const float* scene_spos4,
                           const uint32_t* gidx, const uint32_t* scene_gidx,
                           const uint32_t* cstart, const uint32_t* cend, int n, float* pf4,
                           float* pt4, int* count, float* new_vel4, float* color4) {
  grid_t G;
  memcpy(G.o, grid6, 12); memcpy(G.c, grid6 + 3, 12); memcpy(G.g, dims3, 12);
#pragma omp parallel for schedule(static)
  for (int k = 0; k < n; ++k) {
    v3 pos = xyz(spos4 + 4l * k), vel = xyz(svel4 + 4l * k);
    int gp[3];
    cell_of(&G, pos, gp);
    uint32_t orig = gidx[k];
    int b = rb_idx[orig];
    float ib[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float m = 1.f;
    if (b >= 0) {
      memcpy(ib, inertia9 + 9l * b, 36);
      m = mass[b];
    }
    v3 rel = xyz(rel4 + 4l * orig);
    v3 force = mk3(0.f, 0.f, 0.f), torque = force;
    int ncol = 0;
    uint32_t h = hash3(&G, gp[0], gp[1], gp[2]);
    for (int it = 0; it < 27; ++it) {
      v3 lf = mk3(0.f, 0.f, 0.f), lt = lf;
      if (cstart[h] != 0xffffffffu) {
        for (uint32_t j = cstart[h]; j < cend[h]; ++j) {
          uint32_t o2 = scene_gidx[j];
          v3 q = xyz(scene_spos4 + 4l * j);
          float ra = radius, rb = scene_radii[o2];
          v3 rp = sub(pos, q);
          float dist = sqrtf(dot(rp, rp));
          if (!(dist < ra + rb)) continue;
          ++ncol;
          float t = ra / (ra + rb);
          v3 d = sub(q, pos);
          v3 cp = add(pos, mk3(t * d.x, t * d.y, t * d.z));
          v3 nrm = divs(rp, dist);
          float rv = dot(vel, nrm);
          v3 cm = sub(pos, rel);
          v3 r = mk3(cp.x - cm.x, cp.y - cm.y, cp.z - cm.z);
          v3 a = glm_cross(glm_mv(ib, glm_cross(r, nrm)), r);
          float denom = (a.x * nrm.x + a.y * nrm.y + a.z * nrm.z) + 1.f / m;
          float jj = -(1 + restitution) * rv / denom;
          v3 f = mk3(nrm.x * jj, nrm.y * jj, nrm.z * jj);
          lf = add(lf, f);
          lt = add(lt, cross(r, f));
        }
      }
      force = add(force, lf);
      torque = add(torque, lt);
    }
    if (ncol && color4) st4(color4 + 4l * orig, 0.f, 1.f, 0.f, 0.f);
    if (b == -1) {
      if (new_vel4) {
        float* V = new_vel4 + 4l * orig;
        st4(V, V[0] + force.x, V[1] + force.y, V[2] + force.z, V[3] + 0.f);
      }
    } else {
      st4(pf4 + 4l * orig, force.x, force.y, force.z, 0.f);
      st4(pt4 + 4l * orig, torque.x, torque.y, torque.z, 0.f);
      if (count) count[orig] = ncol;
    }
  }
}

/* Deepest contact with the static scene -- FindAugmentedRealityCollisionsUniformGridCell /
 * Kernel (Kernels/RB_UniformGridKernels.cu:879-1021): 27 neighbour cells, 2r - d deeper than the
 * current contact distance updates distance and point; colour green on any update, else blue. */
void or_ar_find_contacts(const float* grid6, const uint32_t* dims3, float radius,
                         const float* spos4, const float* scene_spos4, const uint32_t* gidx,
                         const uint32_t* scene_gidx, const uint32_t* cstart,
                         const uint32_t* cend, int n, float* contact_distance,
                         int* contact_point, float* color4) {
  grid_t G;
  memcpy(G.o, grid6, 12); memcpy(G.c, grid6 + 3, 12); memcpy(G.g, dims3, 12);
  const float thr = 2 * radius;
#pragma omp parallel for schedule(static)
  for (int k = 0; k < n; ++k) {
    v3 pos = xyz(spos4 + 4l * k);
    int gp[3];
    cell_of(&G, pos, gp);
    uint32_t orig = gidx[k];
    float deepest = contact_distance[orig];
    int best = contact_point[orig], counter = 0;
    for (int z = -1; z <= 1; ++z)
      for (int y = -1; y <= 1; ++y)
        for (int x = -1; x <= 1; ++x) {
          uint32_t h = hash3(&G, gp[0] + x, gp[1] + y, gp[2] + z);
          if (cstart[h] == 0xffffffffu) continue;
          for (uint32_t j = cstart[h]; j < cend[h]; ++j) {
            v3 d = sub(pos, xyz(scene_spos4 + 4l * j));
            float dist = sqrtf(dot(d, d));
            if (thr - dist > deepest) {
              deepest = thr - dist;
              best = (int)scene_gidx[j];
              ++counter;
            }
          }
        }
    contact_distance[orig] = deepest;
    contact_point[orig] = best;
    if (color4) {
      if (counter) st4(color4 + 4l * orig, 0.f, 1.f, 0.f, 0.f);
      else st4(color4 + 4l * orig, 0.f, 0.f, 1.f, 0.f);
    }
  }
}

/* GatherAugmentedRealityCollisions (Particles/updateFunctions.cpp:1511-1578): one contact per
 * particle with a positive contact distance, in particle order. */
long or_gather_static_contacts(float restitution, long n, const int* rb_idx, const float* cms4,
                               const float* vel4, const float* ang4, const float* rel4,
                               const float* scene_normals4, const float* contact_distance,
                               const int* contact_point, float* normal4, float* point4,
                               int* body1, int* body2, float* bias) {
  long c = 0;
  for (long i = 0; i < n; ++i) {
    if (!(contact_distance[i] > 0)) continue;
    int b = rb_idx[i];
    const float* nn = scene_normals4 + 4l * contact_point[i];
    const float *r4 = rel4 + 4 * i, *cm = cms4 + 4l * b;
    v3 v = xyz(vel4 + 4l * b), w = xyz(ang4 + 4l * b);
    float v_rel = dot(add(v, cross(w, xyz(r4))), xyz(nn));
    memcpy(normal4 + 4 * c, nn, 16);
    st4(point4 + 4 * c, r4[0] + cm[0], r4[1] + cm[1], r4[2] + cm[2], r4[3] + cm[3]);
    body1[c] = b;
    body2[c] = -1;
    bias[c] = restitution * v_rel;
    ++c;
  }
  return c;
}

/* ====================================================================================
 * Static scene through a BVH over its point cloud (m leaves; node ids as the Karras build):
 * staticCollideBVHSoARigidBody and FindAugmentedRealityCollisionsBVHKernel
 * (Kernels/RB_BVHKernels.cu:293-442, 920-1023).  The sphere-box test is checkOverlap(float4,
 * AABB, radius) (BVHSource/BVHAuxiliary.cuh:159-175) with a square root rounded toward zero.
 * ==================================================================================== */
static float sqrt_rz(float x) {
  float s = sqrtf(x);
  if ((double)s * (double)s > (double)x) s = nextafterf(s, 0.0f);
  return s;
}
static int sphere_box8(const float* p, const float* b, float r) {
  float xx = fmaxf(b[0], fminf(p[0], b[3]));
  float yy = fmaxf(b[1], fminf(p[1], b[4]));
  float zz = fmaxf(b[2], fminf(p[2], b[5]));
  float d = sqrt_rz((xx - p[0]) * (xx - p[0]) + (yy - p[1]) * (yy - p[1]) +
                    (zz - p[2]) * (zz - p[2]));
  return d < r;
}

/* Per particle: force and torque (rel x force) of every overlapping leaf, the DEM law against a
 * point at rest (collideSpheresBVH, BVHAuxiliary.cuh:97-130), written per particle (a free
 * particle, body -1, gets v + force as its velocity); colour green on a touching leaf.
 * prm = {spring, damping, shear, attraction}. */
void or_collide_bvh_static(const float* prm, float radius, const int* rb_idx, const float* rel4,
                           const float* pos4, float* vel4, const uint8_t* is_leaf,
                           const int* left, const int* right, const float* cms4,
                           const float* bounds8, const float* radii, int m, int n, float* pf4,
                           float* pt4, float* color4) {
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; ++i) {
    const float* qp = pos4 + 4l * i;
    v3 qvel = xyz(vel4 + 4l * i), r3 = xyz(rel4 + 4l * i);
    v3 force = mk3(0.f, 0.f, 0.f), torque = force;
    if (m >= 2) {
      int cap = 256, top = 0;
      int* st = (int*)malloc(sizeof(int) * cap);
      st[top++] = -1;
      int node = m;
      do {
        int lc = left[node], rc = right[node];
        int ol = sphere_box8(qp, bounds8 + 8l * lc, radius);
        int orr = sphere_box8(qp, bounds8 + 8l * rc, radius);
        int ll = is_leaf[lc], rl = is_leaf[rc];
        for (int side = 0; side < 2; ++side) {
          int c = side == 0 ? lc : rc;
          if (!((side == 0 ? ol : orr) && (side == 0 ? ll : rl))) continue;
          const float* cp = cms4 + 4l * c;
          float rc_ = radii[c];
          v3 rp = mk3(cp[0] - qp[0], cp[1] - qp[1], cp[2] - qp[2]);
          float dist = sqrtf(dot(rp, rp));
          v3 f = mk3(0.f, 0.f, 0.f);
          if (dist < radius + rc_)
            f = spring_force(rp, dist, mk3(0.f - qvel.x, 0.f - qvel.y, 0.f - qvel.z),
                             radius + rc_, prm);
          force = add(force, f);
          torque = add(torque, cross(r3, f));
          if (dist < radius + rc_ && color4) st4(color4 + 4l * i, 0.f, 1.f, 0.f, 0.f);
        }
        int tl = ol && !ll, tr = orr && !rl;
        if (!tl && !tr) {
          node = st[--top];
        } else {
          node = tl ? lc : rc;
          if (tl && tr) {
            if (top == cap) { cap *= 2; st = (int*)realloc(st, sizeof(int) * cap); }
            st[top++] = rc;
          }
        }
      } while (node != -1);
      free(st);
    }
    if (rb_idx[i] >= 0) {
      st4(pf4 + 4l * i, force.x, force.y, force.z, 0.f);
      st4(pt4 + 4l * i, torque.x, torque.y, torque.z, 0.f);
    } else {
      st4(vel4 + 4l * i, qvel.x + force.x, qvel.y + force.y, qvel.z + force.z, 0.f);
    }
  }
}

/* Deepest contact through the scene tree: r + radii[point] - |cms[leaf] - p| (four components)
 * deeper than contact_distance[i] records it with the point sorted_idx[leaf]; colour green on a
 * contact, white when none. */
void or_find_contacts_bvh_static(float radius, const float* pos4, const uint8_t* is_leaf,
                                 const int* left, const int* right, const float* cms4,
                                 const float* bounds8, const int* sorted_idx,
                                 const float* radii, int m, int n, float* contact_distance,
                                 int* contact_point, float* color4) {
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < n; ++i) {
    const float* qp = pos4 + 4l * i;
    float deepest = contact_distance[i];
    int best = contact_point[i], ncol = 0;
    if (m >= 2) {
      int cap = 256, top = 0;
      int* st = (int*)malloc(sizeof(int) * cap);
      st[top++] = -1;
      int node = m;
      do {
        int lc = left[node], rc = right[node];
        int ol = sphere_box8(qp, bounds8 + 8l * lc, radius);
        int orr = sphere_box8(qp, bounds8 + 8l * rc, radius);
        int ll = is_leaf[lc], rl = is_leaf[rc];
        for (int side = 0; side < 2; ++side) {
          int c = side == 0 ? lc : rc;
          if (!((side == 0 ? ol : orr) && (side == 0 ? ll : rl))) continue;
          int s_ = sorted_idx[c];
          const float* cp = cms4 + 4l * c;
          float dx = cp[0] - qp[0], dy = cp[1] - qp[1], dz = cp[2] - qp[2], dw = cp[3] - qp[3];
          float dist = sqrtf(dx * dx + dy * dy + dz * dz + dw * dw);
          float thr = radius + radii[s_];
          if (thr - dist > deepest) {
            ++ncol;
            deepest = thr - dist;
            best = s_;
          }
        }
        int tl = ol && !ll, tr = orr && !rl;
        if (!tl && !tr) {
          node = st[--top];
        } else {
          node = tl ? lc : rc;
          if (tl && tr) {
            if (top == cap) { cap *= 2; st = (int*)realloc(st, sizeof(int) * cap); }
            st[top++] = rc;
          }
        }
      } while (node != -1);
      free(st);
    }
    contact_distance[i] = deepest;
    contact_point[i] = best;
    if (color4) {
      if (ncol) st4(color4 + 4l * i, 0.f, 1.f, 0.f, 0.f);
      else st4(color4 + 4l * i, 1.f, 1.f, 1.f, 0.f);
    }
  }
}

/* ---- FP64 oracle of the same physics (summation order free, all-pairs within cells) ---- */
static d3 dk3(double x, double y, double z) { d3 r = {x, y, z}; return r; }
static d3 dadd(d3 a, d3 b) { return dk3(a.x + b.x, a.y + b.y, a.z + b.z); }
static d3 dsub(d3 a, d3 b) { return dk3(a.x - b.x, a.y - b.y, a.z - b.z); }
static d3 dscl(double s, d3 a) { return dk3(s * a.x, s * a.y, s * a.z); }
static double ddot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static d3 dcross(d3 a, d3 b) {
  return dk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static d3 dquat_rotate(const double* q, d3 v) {
  d3 u = dk3(q[0], q[1], q[2]);
  d3 t = dscl(2.0, dcross(u, v));
  return dadd(dadd(v, dscl(q[3], t)), dcross(u, t));
}

/* state arrays in double: bpos4, bquat4, bvel4, bang4 (4 per body); ib9 in double; rel4 in
 * double with the body index in w.  Contacts found by an all-pairs search within the
 * particle's 27 neighbour cells (cell keys from the float32 grid so the candidate sets match). */
int or_step_f64(const double* s15, const double* cell3, int nb, int n, double* bpos4,
                double* bquat4, double* bvel4, double* bang4, const double* mass,
                const double* ib9, const int* off, const double* rel4, int steps,
                double* pforce4_out, double* bforce4_out, double* btorque4_out) {
  const double* bmin = s15; const double* bmax = s15 + 3; const double* gv = s15 + 6;
  double r = s15[9], dt = s15[10], k = s15[11], damping = s15[12], shear = s15[13],
         attraction = s15[14];
  double* pp = (double*)malloc(sizeof(double) * 3 * n);
  double* pv = (double*)malloc(sizeof(double) * 3 * n);
  double* pf = (double*)malloc(sizeof(double) * 4 * n);
  long* ck = (long*)malloc(sizeof(long) * n);
  uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * n);
  uint64_t* kk = (uint64_t*)malloc(sizeof(uint64_t) * n);
  int ok = 1;
  for (int step = 0; step < steps; ++step) {
    for (int i = 0; i < n; ++i) {
      int b = (int)rel4[4l * i + 3];
      d3 rr = dquat_rotate(bquat4 + 4l * b, dk3(rel4[4l * i], rel4[4l * i + 1], rel4[4l * i + 2]));
      d3 p = dadd(dk3(bpos4[4l * b], bpos4[4l * b + 1], bpos4[4l * b + 2]), rr);
      d3 w = dk3(bang4[4l * b], bang4[4l * b + 1], bang4[4l * b + 2]);
      d3 v = dadd(dk3(bvel4[4l * b], bvel4[4l * b + 1], bvel4[4l * b + 2]), dcross(w, rr));
      pp[3 * i] = p.x; pp[3 * i + 1] = p.y; pp[3 * i + 2] = p.z;
      pv[3 * i] = v.x; pv[3 * i + 1] = v.y; pv[3 * i + 2] = v.z;
      long cx = (long)floor((p.x - bmin[0]) / cell3[0]);
      long cy = (long)floor((p.y - bmin[1]) / cell3[1]);
      long cz = (long)floor((p.z - bmin[2]) / cell3[2]);
      /* unbounded cell key: 21 bits per axis, offset to stay positive */
      ck[i] = ((cz + (1 << 20)) << 42) | ((cy + (1 << 20)) << 21) | (cx + (1 << 20));
      kk[i] = (uint64_t)ck[i];
      order[i] = (uint32_t)i;
    }
    lsd_sort_u64(kk, order, n, 63);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
      d3 pos = dk3(pp[3 * i], pp[3 * i + 1], pp[3 * i + 2]);
      d3 vel = dk3(pv[3 * i], pv[3 * i + 1], pv[3 * i + 2]);
      int body = (int)rel4[4l * i + 3];
      long cx = (ck[i] & ((1l << 21) - 1)), cy = (ck[i] >> 21) & ((1l << 21) - 1), cz = ck[i] >> 42;
      d3 F = dk3(0, 0, 0);
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            uint64_t key = (uint64_t)(((cz + dz) << 42) | ((cy + dy) << 21) | (cx + dx));
            long lo = 0, hi = n;
            while (lo < hi) { long mid = (lo + hi) / 2; if (kk[mid] < key) lo = mid + 1; else hi = mid; }
            for (long jj = lo; jj < n && kk[jj] == key; ++jj) {
              int j = (int)order[jj];
              if (j == i || (int)rel4[4l * j + 3] == body) continue;
              d3 rp = dsub(dk3(pp[3 * j], pp[3 * j + 1], pp[3 * j + 2]), pos);
              double dist = sqrt(ddot(rp, rp));
              if (!(dist < 2 * r)) continue;
              d3 nrm = dscl(1.0 / dist, rp);
              d3 rv = dsub(dk3(pv[3 * j], pv[3 * j + 1], pv[3 * j + 2]), vel);
              d3 tv = dsub(rv, dscl(ddot(rv, nrm), nrm));
              d3 f = dscl(-k * (2 * r - dist), nrm);
              f = dadd(f, dscl(damping, rv));
              f = dadd(f, dscl(shear, tv));
              f = dadd(f, dscl(attraction, rp));
              F = dadd(F, f);
            }
          }
      double pc[3] = {pos.x, pos.y, pos.z};
      d3 rv = dk3(-vel.x, -vel.y, -vel.z);
      for (int a = 0; a < 3; ++a)
        for (int side = 0; side < 2; ++side) {
          double d = side == 0 ? pc[a] - bmin[a] : bmax[a] - pc[a];
          if (!(d < r)) continue;
          double sgn = side == 0 ? 1 : -1;
          d3 tv = rv;
          if (a == 0) tv.x = 0; else if (a == 1) tv.y = 0; else tv.z = 0;
          d3 fw = dadd(dscl(damping, rv), dscl(shear, tv));
          double push = sgn * k * (r - d);
          if (a == 0) fw.x += push; else if (a == 1) fw.y += push; else fw.z += push;
          F = dadd(F, fw);
        }
      pf[4l * i] = F.x; pf[4l * i + 1] = F.y; pf[4l * i + 2] = F.z; pf[4l * i + 3] = 0;
    }
    for (int b = 0; b < nb; ++b) {
      d3 F = dk3(0, 0, 0), T = dk3(0, 0, 0);
      const double* q = bquat4 + 4l * b;
      for (int i = off[b]; i < off[b + 1]; ++i) {
        d3 f = dk3(pf[4l * i], pf[4l * i + 1], pf[4l * i + 2]);
        F = dadd(F, f);
        T = dadd(T, dcross(dquat_rotate(q, dk3(rel4[4l * i], rel4[4l * i + 1], rel4[4l * i + 2])), f));
      }
      if (bforce4_out) { double* o = bforce4_out + 4l * b; o[0] = F.x; o[1] = F.y; o[2] = F.z; o[3] = 0; }
      if (btorque4_out) { double* o = btorque4_out + 4l * b; o[0] = T.x; o[1] = T.y; o[2] = T.z; o[3] = 0; }
      double m = mass[b];
      double* V = bvel4 + 4l * b; double* W = bang4 + 4l * b; double* P = bpos4 + 4l * b;
      double* Q = bquat4 + 4l * b;
      for (int a = 0; a < 3; ++a) V[a] += dt * (gv[a] + (a == 0 ? F.x : a == 1 ? F.y : F.z) / m);
      double qc[4] = {-Q[0], -Q[1], -Q[2], Q[3]};
      d3 tb = dquat_rotate(qc, T);
      const double* I = ib9 + 9l * b;
      d3 lb = dk3(I[0] * tb.x + I[3] * tb.y + I[6] * tb.z, I[1] * tb.x + I[4] * tb.y + I[7] * tb.z,
                  I[2] * tb.x + I[5] * tb.y + I[8] * tb.z);
      d3 dw = dquat_rotate(Q, lb);
      W[0] += dt * dw.x; W[1] += dt * dw.y; W[2] += dt * dw.z;
      for (int a = 0; a < 3; ++a) P[a] += dt * V[a];
      double qd[4];
      qd[3] = -W[0] * Q[0] - W[1] * Q[1] - W[2] * Q[2];
      qd[0] = W[0] * Q[3] + W[1] * Q[2] - W[2] * Q[1];
      qd[1] = W[1] * Q[3] + W[2] * Q[0] - W[0] * Q[2];
      qd[2] = W[2] * Q[3] + W[0] * Q[1] - W[1] * Q[0];
      double nq[4];
      for (int c = 0; c < 4; ++c) nq[c] = Q[c] + 0.5 * dt * qd[c];
      double len = sqrt(nq[0] * nq[0] + nq[1] * nq[1] + nq[2] * nq[2] + nq[3] * nq[3]);
      for (int c = 0; c < 4; ++c) Q[c] = nq[c] / len;
      if (!isfinite(P[0] + P[1] + P[2] + V[0] + V[1] + V[2] + W[0] + W[1] + W[2])) ok = 0;
    }
  }
  if (pforce4_out) memcpy(pforce4_out, pf, sizeof(double) * 4 * n);
  free(pp); free(pv); free(pf); free(ck); free(order); free(kk);
  return ok;
}

/* ====================================================================================
 * (a3) integrateRigidBody (Kernels/rigidBodyKernels.cu:40-166), momentum form.
 * ==================================================================================== */
void or_integrate_momentum(float* cms4, float* vel4, float* force4, float* ang4, float* quat4,
                           float* torque4, float* angmom4, float* linmom4, const float* ib9,
                           float* cur9, float* acc3, float dt, const float* radii,
                           const float* mass, const float* mn3, const float* mx3,
                           const float* gravity3, float bdamp, float gdamp, int nb) {
  for (int b = 0; b < nb; ++b) {
    float* L = linmom4 + 4l * b;
    const float* F = force4 + 4l * b;
    float l[4] = {L[0] + F[0] * dt, L[1] + F[1] * dt, L[2] + F[2] * dt, L[3] + F[3] * dt};
    l[0] = l[0] + gravity3[0] * dt; l[1] = l[1] + gravity3[1] * dt;
    l[2] = l[2] + gravity3[2] * dt; l[3] = l[3] + 0.f * dt;
    float mx[3] = {(float)((double)mx3[0] + 0.1), (float)((double)mx3[1] + 0.1), (float)((double)mx3[2] + 0.1)};
    float mn[3] = {(float)((double)mn3[0] - 0.1), (float)((double)mn3[1] - 0.1), mn3[2] - 1};
    float* P = cms4 + 4l * b;
    float p[4] = {P[0], P[1], P[2], P[3]};
    float m = mass[b], r = radii[b];
    if (p[0] > mx[0] - r) { p[0] = mx[0] - r; l[0] *= bdamp; }
    if (p[0] < mn[0] + r) { p[0] = mn[0] + r; l[0] *= bdamp; }
    if (p[1] > mx[1] - r && l[1] > 0) { p[1] = mx[1] - 2 * r; l[1] *= bdamp; }
    if (p[1] < mn[1] + r) { p[1] = mn[1] + r; l[1] *= bdamp; }
    if (p[2] > mx[2] - r) { p[2] = mx[2] - r; l[2] *= bdamp; }
    if (p[2] < mn[2] + r) { p[2] = mn[2] + r; l[2] *= bdamp; }
    for (int c = 0; c < 4; ++c) l[c] = l[c] * gdamp;
    float v[4] = {l[0] * m, l[1] * m, l[2] * m, l[3] * m};
    memcpy(L, l, 16);
    for (int c = 0; c < 4; ++c) p[c] = p[c] + v[c] * dt;
    p[3] = 0.f; v[3] = 0.f;
    memcpy(P, p, 16);
    memcpy(vel4 + 4l * b, v, 16);
    memset(force4 + 4l * b, 0, 16);
    v4 q = ld4(quat4 + 4l * b);
    float R[9], RI[9], Rt[9], C[9];
    glm_mat3_cast(q, R);
    glm_mm(R, ib9 + 9l * b, RI);
    for (int c = 0; c < 3; ++c) for (int rr = 0; rr < 3; ++rr) Rt[c * 3 + rr] = R[rr * 3 + c];
    glm_mm(RI, Rt, C);
    float* A = angmom4 + 4l * b;
    const float* T = torque4 + 4l * b;
    float am[4] = {A[0] + T[0] * dt, A[1] + T[1] * dt, A[2] + T[2] * dt, A[3] + T[3] * dt};
    v3 cm3 = mk3(am[0], am[1], am[2]);
    v3 nv = glm_mv(C, cm3);
    v3 acc = glm_mv(C, glm_cross(cm3, nv));
    v4 wq = {nv.x, nv.y, nv.z, 0.f};
    v4 qd = glm_qmul(wq, q);
    qd.x = qd.x / 2.f; qd.y = qd.y / 2.f; qd.z = qd.z / 2.f; qd.w = qd.w / 2.f;
    q.x = q.x + qd.x * dt; q.y = q.y + qd.y * dt; q.z = q.z + qd.z * dt; q.w = q.w + qd.w * dt;
    q = glm_qnormalize(q);
    nv = mk3(nv.x - acc.x * dt, nv.y - acc.y * dt, nv.z - acc.z * dt);
    if (acc3) { acc3[3 * b] = acc.x; acc3[3 * b + 1] = acc.y; acc3[3 * b + 2] = acc.z; }
    memcpy(cur9 + 9l * b, C, 36);
    memcpy(A, am, 16);
    st4(quat4 + 4l * b, q.x, q.y, q.z, q.w);
    st4(ang4 + 4l * b, nv.x, nv.y, nv.z, 0.f);
    memset(torque4 + 4l * b, 0, 16);
  }
}

/* (a5) integrate_functor (Kernels/particleKernels.cu:50-128), free particles only. */
void or_integrate_particles(float* pos4, float* vel4, const int* rb_idx, int n, float dt,
                            const float* mn3, const float* mx3, const float* gravity3,
                            float gdamp, float bdamp, float r) {
  float mx[3] = {(float)((double)mx3[0] + 0.01), (float)((double)mx3[1] + 0.01), (float)((double)mx3[2] + 0.01)};
  float mn[3] = {(float)((double)mn3[0] - 0.01), (float)((double)mn3[1] - 0.01), (float)((double)mn3[2] - 0.01)};
  for (int i = 0; i < n; ++i) {
    if (rb_idx[i] >= 0) continue;
    float* P = pos4 + 4l * i;
    float* V = vel4 + 4l * i;
    v3 p = xyz(P), v = xyz(V);
    v = add(v, mk3(gravity3[0] * dt, gravity3[1] * dt, gravity3[2] * dt));
    v = mk3(v.x * gdamp, v.y * gdamp, v.z * gdamp);
    p = add(p, mk3(v.x * dt, v.y * dt, v.z * dt));
    if (p.x > mx[0] - r) { p.x = mx[0] - r; v.x *= bdamp; }
    if (p.x < mn[0] + r) { p.x = mn[0] + r; v.x *= bdamp; }
    if (p.y > mx[1] - r && v.y > 0) { p.y = mx[1] - r; v.y *= bdamp; }
    if (p.z > mx[2] - r) { p.z = mx[2] - r; v.z *= bdamp; }
    if (p.z < mn[2] + r) { p.z = mn[2] + r; v.z *= bdamp; }
    if (p.y < mn[1] + r) { p.y = mn[1] + r; v.y *= bdamp; }
    P[0] = p.x; P[1] = p.y; P[2] = p.z;
    V[0] = v.x; V[1] = v.y; V[2] = v.z;
  }
}

/* collideD / collideCell / collideSpheres (Kernels/particleKernels.cu:261-406). */
void or_collide_grid_particles(const float* grid6, const uint32_t* dims3, const float* prm5,
                               const int* rb_idx, const float* spos4, const float* svel4,
                               const float* rel4, const uint32_t* gidx, const uint32_t* cstart,
                               const uint32_t* cend, long n, float* p_force4, float* p_torque4,
                               float* new_vel4) {
  grid_t G;
  memcpy(G.o, grid6, 12); memcpy(G.c, grid6 + 3, 12); memcpy(G.g, dims3, 12);
  const float cd = prm5[4] + prm5[4];
#pragma omp parallel for schedule(static)
  for (long index = 0; index < n; ++index) {
    v3 pos = xyz(spos4 + 4 * index), vel = xyz(svel4 + 4 * index);
    int gp[3];
    cell_of(&G, pos, gp);
    uint32_t orig = gidx[index];
    int body = rb_idx[orig];
    v3 r3 = xyz(rel4 + 4l * orig);
    v3 force = mk3(0.f, 0.f, 0.f), torque = mk3(0.f, 0.f, 0.f);
    for (int z = -1; z <= 1; ++z)
      for (int y = -1; y <= 1; ++y)
        for (int x = -1; x <= 1; ++x) {
          v3 cf = mk3(0.f, 0.f, 0.f);
          uint32_t h = hash3(&G, gp[0] + x, gp[1] + y, gp[2] + z);
          uint32_t s = cstart[h];
          if (s != EMPTY) {
            uint32_t e = cend[h];
            for (uint32_t j = s; j < e; ++j) {
              if (!(j != (uint32_t)index && (body != rb_idx[gidx[j]] || body == -1))) continue;
              v3 rp = sub(xyz(spos4 + 4l * j), pos);
              float dist = sqrtf(dot(rp, rp));
              v3 f = mk3(0.f, 0.f, 0.f);
              if (dist < cd) f = spring_force(rp, dist, sub(xyz(svel4 + 4l * j), vel), cd, prm5);
              cf = add(cf, f);
            }
          }
          force = add(force, cf);
          torque = add(torque, cross(r3, cf));
        }
    if (body == -1) {
      if (new_vel4) st4(new_vel4 + 4l * orig, vel.x + force.x, vel.y + force.y, vel.z + force.z, 0.f);
    } else {
      st4(p_force4 + 4l * orig, force.x, force.y, force.z, 0.f);
      st4(p_torque4 + 4l * orig, torque.x, torque.y, torque.z, 0.f);
    }
  }
}

/* (a17) ReduceRigidBodyVariables (Kernels/rigidBodyKernels.cu:861-1043): += fixed-order sums;
 * returns 0 when a sum is not finite (the reference's *toExit). */
int or_reduce_rbvars(const float* pf4, const float* pt4, const int* starts, const int* counts,
                     int nb, float* bf4, float* bt4) {
  int ok = 1;
  for (int b = 0; b < nb; ++b) {
    int s = starts[b], c = counts[b];
    v3* f = (v3*)malloc(sizeof(v3) * (c + 1));
    v3* t = (v3*)malloc(sizeof(v3) * (c + 1));
    for (int i = 0; i < c; ++i) { f[i] = xyz(pf4 + 4l * (s + i)); t[i] = xyz(pt4 + 4l * (s + i)); }
    v3 F = warp_sum(f, c), T = warp_sum(t, c);
    free(f); free(t);
    if (!isfinite(F.x + F.y + F.z) || !isfinite(T.x + T.y + T.z)) ok = 0;
    float* o = bf4 + 4l * b;
    o[0] = o[0] + F.x; o[1] = o[1] + F.y; o[2] = o[2] + F.z;
    o = bt4 + 4l * b;
    o[0] = o[0] + T.x; o[1] = o[1] + T.y; o[2] = o[2] + T.z;
  }
  return ok;
}

/* ====================================================================================
 * Sequential-impulse path (updateUniformGridSIS, RigidBodies/UniformGridUpdate.cpp:734-815).
 * ==================================================================================== */

/* FindRigidBodyCollisionsUniformGridCell / Kernel (Kernels/RB_UniformGridKernels.cu:731-842):
 * per sorted particle, the deepest penetration by a particle of another body, above the running
 * maximum contact_distance[original] (re-read per neighbour cell). */
void or_find_contacts_grid(const float* grid6, const uint32_t* dims3, float radius,
                           const int* rb_idx, const float* spos4, const uint32_t* gidx,
                           const uint32_t* cstart, const uint32_t* cend, long n,
                           float* contact_distance, int* colliding_body,
                           int* colliding_particle) {
  grid_t G;
  memcpy(G.o, grid6, 12); memcpy(G.c, grid6 + 3, 12); memcpy(G.g, dims3, 12);
  const float threshold = 2 * radius;
  for (long index = 0; index < n; ++index) {
    v3 pos = xyz(spos4 + 4 * index);
    int gp[3];
    cell_of(&G, pos, gp);
    uint32_t orig = gidx[index];
    int body = rb_idx[orig];
    for (int z = -1; z <= 1; ++z)
      for (int y = -1; y <= 1; ++y)
        for (int x = -1; x <= 1; ++x) {
          uint32_t h = hash3(&G, gp[0] + x, gp[1] + y, gp[2] + z);
          uint32_t st = cstart[h];
          float best = contact_distance[orig];
          if (st == EMPTY) continue;
          uint32_t en = cend[h];
          for (uint32_t j = st; j < en; ++j) {
            int o2 = (int)gidx[j];
            int b2 = rb_idx[o2];
            if (j == (uint32_t)index || b2 == body) continue;
            v3 d = sub(pos, xyz(spos4 + 4 * j));
            float dist = sqrtf(dot(d, d));
            if (threshold - dist > best) {
              best = threshold - dist;
              contact_distance[orig] = best;
              colliding_particle[orig] = o2;
              colliding_body[orig] = b2;
            }
          }
        }
  }
}

/* GatherRigidBodyCollisions (Particles/updateFunctions.cpp:1431-1500) with findExactContactPoint
 * (Particles/CPU_Engine.cpp:461-473): float4 arithmetic, normalize = v * (1 / sqrt(dot4)). */
long or_gather_contacts(float radius, float restitution, long n, const int* rb_idx,
                        const float* cms4, const float* vel4, const float* ang4,
                        const float* rel4, const float* contact_distance,
                        const int* colliding_body, const int* colliding_particle,
                        float* normal4, float* point4, int* body1, int* body2, float* bias) {
  long c = 0;
  for (long i = 0; i < n; ++i) {
    if (!(contact_distance[i] > 0)) continue;
    int b = rb_idx[i], j = colliding_particle[i], b2 = colliding_body[i];
    const float *cm1 = cms4 + 4 * b, *cm2 = cms4 + 4 * b2, *r1 = rel4 + 4 * (long)i,
                *r2 = rel4 + 4 * (long)j;
    float p1[4], p2[4], cp[4], d[4], cn[4];
    for (int k = 0; k < 4; ++k) {
      p1[k] = cm1[k] + r1[k];
      p2[k] = cm2[k] + r2[k];
    }
    float t = radius / (radius + radius);
    for (int k = 0; k < 4; ++k) {
      cp[k] = p1[k] + (p2[k] - p1[k]) * t;
      d[k] = p2[k] - p1[k];
    }
    float inv = 1.0f / sqrtf(d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + d[3] * d[3]);
    for (int k = 0; k < 4; ++k) cn[k] = d[k] * inv * (-1.f);
    v3 n3 = mk3(cn[0], cn[1], cn[2]);
    v3 v1 = xyz(vel4 + 4 * b), w1 = xyz(ang4 + 4 * b);
    v3 v2 = xyz(vel4 + 4 * b2), w2 = xyz(ang4 + 4 * b2);
    float v_rel = dot(add(v1, cross(w1, xyz(r1))), n3) - dot(add(v2, cross(w2, xyz(r2))), n3);
    memcpy(normal4 + 4 * c, cn, 16);
    memcpy(point4 + 4 * c, cp, 16);
    body1[c] = b;
    body2[c] = b2;
    bias[c] = restitution * v_rel;
    ++c;
  }
  return c;
}

static float clampf_(float v, float lo, float hi) { return v < lo ? lo : (v > hi ? hi : v); }
static v3 gnormalize_(v3 v) {
  float inv = 1.0f / sqrtf(dot(v, v));
  return mk3(v.x * inv, v.y * inv, v.z * inv);
}

/* SequentialImpulseSolver (Particles/updateFunctions.cpp:1580-1874), the host loop as written:
 * float arithmetic, the abs(x) < 0.00001 / 0.0001 tests in double (float promoted), accumulated
 * impulse clamped to [0, 100]. */
void or_sequential_impulse(long count, const float* normal4, const float* point4,
                           const int* body1, const int* body2, const float* bias,
                           float* acc_impulse, float* acc_friction, float* acc_friction2,
                           const float* cms4, float* vel4, float* ang4, const float* inertia9,
                           const float* mass, int iterations, float ar_friction,
                           float rb_friction, float gravity_y) {
  const float upper = 100.f, g = fabsf(gravity_y);
  for (int it = 0; it < iterations; ++it)
    for (long c = 0; c < count; ++c) {
      v3 n = xyz(normal4 + 4 * c);
      const float* pt = point4 + 4 * c;
      int i1 = body1[c], i2 = body2[c];
      const float* cm1 = cms4 + 4 * i1;
      v3 p1 = mk3(pt[0] - cm1[0], pt[1] - cm1[1], pt[2] - cm1[2]);
      const float* I1 = inertia9 + 9 * i1;
      float m1 = mass[i1];
      v3 v1 = xyz(vel4 + 4 * i1), w1 = xyz(ang4 + 4 * i1);
      if (i2 == -1) {
        float mc = 1 / m1 + dot(glm_cross(glm_mv(I1, glm_cross(p1, n)), p1), n);
        if ((double)fabsf(mc) < 0.00001) mc = 1.f;
        float v_rel = dot(add(v1, glm_cross(w1, p1)), n);
        float corr = -(v_rel + bias[c]) / mc;
        float acc = acc_impulse[c];
        float tmp = clampf_(acc + corr, 0.f, upper);
        corr = tmp - acc;
        acc_impulse[c] = tmp;
        float bound = ar_friction * mc * g;
        v3 vel = add(v1, glm_cross(w1, p1));
        v3 t1 = mk3(1.f, 0.f, 0.f);
        if ((double)fabsf(t1.x - n.x) < 0.0001) t1 = mk3(0.f, 1.f, 0.f);
        else if ((double)fabsf(t1.x + n.x) < 0.0001) t1 = mk3(0.f, 1.f, 0.f);
        t1 = gnormalize_(sub(t1, scl(dot(t1, n), n)));
        float k1 = 1 / m1 + dot(glm_cross(glm_mv(I1, glm_cross(p1, t1)), p1), t1);
        float cf1 = -dot(vel, t1) / k1;
        float a1 = acc_friction[c];
        float f1 = clampf_(a1 + cf1, -bound, bound);
        cf1 = f1 - a1;
        acc_friction[c] = f1;
        v3 t2 = gnormalize_(glm_cross(t1, n));
        float k2 = 1 / m1 + dot(glm_cross(glm_mv(I1, glm_cross(p1, t2)), p1), t2);
        float cf2 = -dot(vel, t2) / k2;
        float a2 = acc_friction2[c];
        float f2 = clampf_(a2 + cf2, -bound, bound);
        cf2 = f2 - a2;
        acc_friction2[c] = f2;
        v3 imp = add(add(scl(corr, n), scl(cf1, t1)), scl(cf2, t2));
        v1 = add(v1, divs(imp, m1));
        w1 = add(w1, glm_mv(I1, glm_cross(p1, imp)));
        st4(vel4 + 4 * i1, v1.x, v1.y, v1.z, 0.f);
        st4(ang4 + 4 * i1, w1.x, w1.y, w1.z, 0.f);
        continue;
      }
      const float* cm2 = cms4 + 4 * i2;
      v3 p2 = mk3(pt[0] - cm2[0], pt[1] - cm2[1], pt[2] - cm2[2]);
      const float* I2 = inertia9 + 9 * i2;
      float m2 = mass[i2];
      v3 v2 = xyz(vel4 + 4 * i2), w2 = xyz(ang4 + 4 * i2);
      float mc = 1 / m1 + 1 / m2 + dot(glm_cross(glm_mv(I1, glm_cross(p1, n)), p1), n) +
                 dot(glm_cross(glm_mv(I2, glm_cross(p2, n)), p2), n);
      if ((double)fabsf(mc) < 0.00001) mc = 1.f;
      float v_rel = dot(add(v1, glm_cross(w1, p1)), n) - dot(add(v2, glm_cross(w2, p2)), n);
      float corr = -(v_rel + bias[c]) / mc;
      float acc = acc_impulse[c];
      float tmp = clampf_(acc + corr, 0.f, upper);
      corr = tmp - acc;
      acc_impulse[c] = tmp;
      float bound = rb_friction * mc * g;
      v3 vel = add(add(add(scl(-1.f, v1), glm_cross(w1, p1)), v2), glm_cross(w2, p2));
      v3 t1 = mk3(1.f, 0.f, 0.f);
      if ((double)fabsf(t1.x - n.x) < 0.0001) t1 = mk3(0.f, 1.f, 0.f);
      t1 = gnormalize_(sub(t1, scl(dot(t1, n), n)));
      float k1 = (1 / m1 + dot(glm_cross(glm_mv(I1, glm_cross(p1, t1)), p1), t1)) +
                 (1 / m2 + dot(glm_cross(glm_mv(I2, glm_cross(p2, t1)), p2), t1));
      float cf1 = -dot(vel, t1) / k1;
      acc_friction[c] = clampf_(acc_friction[c] + cf1, -bound, bound);
      v3 t2 = gnormalize_(glm_cross(t1, n));
      float k2 = (1 / m1 + dot(glm_cross(glm_mv(I1, glm_cross(p1, t2)), p1), t2)) +
                 (1 / m2 + dot(glm_cross(glm_mv(I2, glm_cross(p2, t2)), p2), t2));
      float cf2 = -dot(vel, t2) / k2;
      acc_friction2[c] = clampf_(acc_friction2[c] + cf2, -bound, bound);
      v3 imp = scl(corr, n);
      v1 = add(v1, divs(imp, m1));
      w1 = add(w1, glm_mv(I1, glm_cross(p1, imp)));
      st4(vel4 + 4 * i1, v1.x, v1.y, v1.z, 0.f);
      st4(ang4 + 4 * i1, w1.x, w1.y, w1.z, 0.f);
      v2 = sub(v2, divs(imp, m2));
      w2 = sub(w2, glm_mv(I2, glm_cross(p2, imp)));
      st4(vel4 + 4 * i2, v2.x, v2.y, v2.z, 0.f);
      st4(ang4 + 4 * i2, w2.x, w2.y, w2.z, 0.f);
    }
}

/* ---- depth-camera ingestion (Kernels/customRangeImageLoader.cu) ----------------------------
 * RGBDloader (:14-113) and computeNormals (:122-177), per pixel in the reference's arithmetic
 * order; glm 0.9.7 mat4 * vec4 pairs (m0 v0 + m1 v1) + (m2 v2 + m3 v3); normalize takes
 * 1 / sqrtf (helper_math's host rsqrtf, glm's inversesqrt). */
static void or_mat4_mul_(const float m[16], const float v[4], float out[4]) {
  for (int i = 0; i < 4; ++i) {
    const float a0 = m[0 * 4 + i] * v[0] + m[1 * 4 + i] * v[1];
    const float a1 = m[2 * 4 + i] * v[2] + m[3 * 4 + i] * v[3];
    out[i] = a0 + a1;
  }
}

void or_range_cloud(const uint16_t* depth, int w, int h, const float* cam16, float radius,
                    float* pos4, float* radii, float* vao5) {
  float t[16];  /* transpose (column-major in, column-major out) */
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r) t[4 * c + r] = cam16[4 * r + c];
  const float fx = (float)517.3, fy = (float)516.5, cx = (float)318.6, cy = (float)255.3;
  const float gx0 = (float)0.478957, gy0 = (float)-8.010560, gz0 = (float)4.166928;
  const float inv = 1.0f / sqrtf(gx0 * gx0 + gy0 * gy0 + gz0 * gz0);
  const float gx = gx0 * inv, gy = gy0 * inv, gz = gz0 * inv;
  const float grav[16] = {1.f, 0.f, 0.f, 0.f, -gx, -gy, -gz, 0.f,
                          0.f, gz, -gy, 0.f, 0.f, 0.f, 0.f, 1.f};
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      const long index = (long)y * w + x;
      if (index > (long)(w - 1) * (h - 1)) continue;
      float pz = (float)depth[index];
      pz /= 5000.f;
      radii[index] = radius;
      if ((double)pz < 0.01) pz = -1000.f;
      const float px = pz * ((float)x - cx) / fx;
      const float py = pz * ((float)y - cy) / fy;
      const float v[4] = {px, py, pz, 0.f};
      float a[4], b[4];
      or_mat4_mul_(t, v, a);
      or_mat4_mul_(grav, a, b);
      const float ox = b[0], oy = -b[1], oz = -b[2];
      if (vao5) {
        vao5[5 * index] = ox;
        vao5[5 * index + 1] = oy;
        vao5[5 * index + 2] = oz;
        vao5[5 * index + 3] = (float)x / (float)w;
        vao5[5 * index + 4] = (float)y / (float)h;
      }
      pos4[4 * index] = ox;
      pos4[4 * index + 1] = oy;
      pos4[4 * index + 2] = oz;
      pos4[4 * index + 3] = 0.f;
    }
}

void or_range_normals(const float* pos4, int w, int h, float* norm4) {
  for (int y = 1; y < h - 1; ++y)
    for (int x = 1; x < w - 1; ++x) {
      const float* up = pos4 + 4 * ((long)(y - 1) * w + x);
      const float* right = pos4 + 4 * ((long)y * w + x + 1);
      const float* down = pos4 + 4 * ((long)(y + 1) * w + x);
      const float* left = pos4 + 4 * ((long)y * w + x - 1);
      const float dx[3] = {right[0] - left[0], right[1] - left[1], right[2] - left[2]};
      const float dy[3] = {down[0] - up[0], down[1] - up[1], down[2] - up[2]};
      const float c[3] = {dy[1] * dx[2] - dy[2] * dx[1], dy[2] * dx[0] - dy[0] * dx[2],
                          dy[0] * dx[1] - dy[1] * dx[0]};
      const float inv = 1.0f / sqrtf(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
      float* o = norm4 + 4 * ((long)y * w + x);
      o[0] = c[0] * inv;
      o[1] = c[1] * inv;
      o[2] = c[2] * inv;
      o[3] = 0.f;
    }
}
