// Device-side scene table and the PHYSICAL-mode per-particle / per-body math of the fused
// step.  Every function here is mirrored operation for operation by the oracle
// (oracle/oracle.c, or_step / or_step_bvh), which is what makes stepped states bit-identical.
#pragma once
#include "ar_internal.cuh"
#include "ar_glm.cuh"

namespace ar_pipe {

// One scene in a batch: its parameters, its place in the batch's concatenated index spaces
// and pointers to its resident arrays.
struct SceneDev {
  float bmin[3], bmax[3];   // box walls
  float g[3];               // gravity
  float r, dt, k, damping, shear, attraction;
  float origin[3], cell[3]; // grid
  float inv_cell[3];        // 1 / cell, used when every cell edge is a power of two
  int cell_pow2;            // (then x * inv_cell == x / cell exactly)
  uint32_t gx, gy, gz;      // cells per axis (powers of two)
  uint32_t lx, ly;          // log2 gx, log2 gy
  uint32_t cell_base;       // first cell of the scene in the batch's global cell space
  int poff, boff, n, nb;    // first particle / body in the batch, counts
  long long end_step;       // last batch step that integrates the scene (then it is frozen)
  float4* pos;              // body centre (w unused)
  float4* quat;             // (x, y, z, w)
  float4* vel;
  float4* ang;
  const float* mass;
  const float* inv_inertia;  // body frame, glm::mat3 layout, 9 per body
  const int32_t* offsets;    // B+1
  const float4* rel;         // body-frame offset, w = local body index (int bits)
  float4* bforce;            // last step's per-body totals
  float4* btorque;
  // static point cloud of the scene (null: none): its points sorted by cell of this scene's
  // grid, with their normals, and {first, end} of every cell's points by local cell key
  const uint2* cloud_cells;
  const float4* cloud_pos;
  const float4* cloud_norm;
};

__host__ __device__ __forceinline__ int3 cell_of(const SceneDev& s, float3 p) {
  if (s.cell_pow2)  // division by a power of two is the multiplication by its inverse
    return make_int3((int)floorf((p.x - s.origin[0]) * s.inv_cell[0]),
                     (int)floorf((p.y - s.origin[1]) * s.inv_cell[1]),
                     (int)floorf((p.z - s.origin[2]) * s.inv_cell[2]));
  return make_int3((int)floorf((p.x - s.origin[0]) / s.cell[0]),
                   (int)floorf((p.y - s.origin[1]) / s.cell[1]),
                   (int)floorf((p.z - s.origin[2]) / s.cell[2]));
}
__host__ __device__ __forceinline__ uint32_t cell_key(const SceneDev& s, int3 c) {
  const uint32_t x = (uint32_t)c.x & (s.gx - 1), y = (uint32_t)c.y & (s.gy - 1),
                 z = (uint32_t)c.z & (s.gz - 1);
  return s.cell_base + (z * s.gy * s.gx + y * s.gx + x);
}

// World-frame lever arm, position and velocity of a particle of a body with centre c,
// orientation q, velocity v and angular velocity w.
__host__ __device__ __forceinline__ void repose(float4 q, float4 c, float4 v, float4 w,
                                                float3 rel, float3* r, float3* p, float3* pv) {
  *r = ar::quat_rotate(q, rel);
  *p = ar::add(ar::xyz(c), *r);
  *pv = ar::add(ar::xyz(v), ar::cross(ar::xyz(w), *r));
}

// Box walls as DEM contacts with a static plane: for each plane the particle penetrates
// (centre closer than r), spring k * depth along the inward normal, dashpot on the full
// relative velocity (-v) and shear on its tangential part -- the particle-particle law with
// the plane as a body at rest.  Planes in order -x, +x, -y, +y, -z, +z.
__host__ __device__ __forceinline__ float3 wall_force(const SceneDev& s, float3 p, float3 v) {
  float3 f = ar::mk3(0.f, 0.f, 0.f);
  const float pc[3] = {p.x, p.y, p.z};
  const float3 rv = ar::mk3(-v.x, -v.y, -v.z);
  for (int a = 0; a < 3; ++a) {
    for (int side = 0; side < 2; ++side) {
      const float d = side == 0 ? pc[a] - s.bmin[a] : s.bmax[a] - pc[a];
      if (!(d < s.r)) continue;
      const float sgn = side == 0 ? 1.f : -1.f;
      float3 tv = rv;
      if (a == 0) tv.x = 0.f; else if (a == 1) tv.y = 0.f; else tv.z = 0.f;
      float3 fw = ar::add(ar::scl(s.damping, rv), ar::scl(s.shear, tv));
      const float push = sgn * (s.k * (s.r - d));
      if (a == 0) fw.x = fw.x + push; else if (a == 1) fw.y = fw.y + push; else fw.z = fw.z + push;
      f = ar::add(f, fw);
    }
  }
  return f;
}

// Semi-implicit Euler update of one body from its summed force F and torque T:
//   v += dt (g + F/m);  w += dt R Ib^-1 R^T T;  x += dt v;  q = normalise(q + dt/2 (w,0) q).
// Returns false when the new state is not finite.
__host__ __device__ __forceinline__ bool integrate_body(const SceneDev& s, float3 F, float3 T,
                                                        float m, const float* ib, float4* pos,
                                                        float4* quat, float4* vel,
                                                        float4* ang) {
  const float dt = s.dt;
  float4 q = *quat, c = *pos, v = *vel, w = *ang;
  const float3 acc = ar::add(ar::mk3(s.g[0], s.g[1], s.g[2]), ar::divs(F, m));
  const float3 nv = ar::add(ar::xyz(v), ar::scl(dt, acc));
  const float4 qc = make_float4(-q.x, -q.y, -q.z, q.w);
  const float3 tb = ar::quat_rotate(qc, T);          // R^T T
  const float3 lb = ar_glm::mv(ib, tb);              // Ib^-1 R^T T
  const float3 dw = ar::quat_rotate(q, lb);          // R Ib^-1 R^T T
  const float3 nw = ar::add(ar::xyz(w), ar::scl(dt, dw));
  const float3 nc = ar::add(ar::xyz(c), ar::scl(dt, nv));
  const float4 qd = ar_glm::qmul(make_float4(nw.x, nw.y, nw.z, 0.f), q);
  const float h = 0.5f * dt;
  float4 nq = make_float4(q.x + h * qd.x, q.y + h * qd.y, q.z + h * qd.z, q.w + h * qd.w);
  const float inv = 1.f / sqrtf(((nq.x * nq.x + nq.y * nq.y) + nq.z * nq.z) + nq.w * nq.w);
  nq = make_float4(nq.x * inv, nq.y * inv, nq.z * inv, nq.w * inv);
  *pos = make_float4(nc.x, nc.y, nc.z, c.w);
  *vel = make_float4(nv.x, nv.y, nv.z, v.w);
  *ang = make_float4(nw.x, nw.y, nw.z, w.w);
  *quat = nq;
  const float chk = nc.x + nc.y + nc.z + nv.x + nv.y + nv.z + nw.x + nw.y + nw.z + nq.x + nq.y +
                    nq.z + nq.w;
  return isfinite(chk);
}

}  // namespace ar_pipe
