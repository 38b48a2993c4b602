// DEM pair arithmetic shared by the grid and BVH kernels.  Each function evaluates its
// expression in the reference's operation order (see the cited lines); with the library's
// -fmad=false build every rounding is the same as in the reference's source read literally.
#pragma once
#include "ar_internal.cuh"

namespace ar_dem {

// Canonical contact test: |pb - pa| < two_r with |v| = sqrtf(dot(v, v)) -- the test of
// FindAndHandleRigidBodyCollisionsUniformGridCell (RigidBodies/UniformGridDEM.cu:96-98) and
// collideStaticSpheresBVH (Kernels/RB_BVHKernels.cu:31-38).  Symmetric in (a, b).
__host__ __device__ __forceinline__ bool touching(float3 pa, float3 pb, float two_r) {
  float3 rp = ar::sub(pb, pa);
  return sqrtf(ar::dot(rp, rp)) < two_r;
}

// Spring-dashpot-shear-attraction force on A from B, without the distance test
// (UniformGridDEM.cu:102-118): rp = pB - pA, d = |rp|.
__host__ __device__ __forceinline__ float3 spring_force(float3 rp, float dist, float3 rv,
                                                        float contact, float spring,
                                                        float damping, float shear,
                                                        float attraction) {
  float3 nrm = ar::divs(rp, dist);
  float3 tv = ar::sub(rv, ar::scl(ar::dot(rv, nrm), nrm));
  float3 f = ar::scl(-spring * (contact - dist), nrm);
  f = ar::add(f, ar::scl(damping, rv));
  f = ar::add(f, ar::scl(shear, tv));
  f = ar::add(f, ar::scl(attraction, rp));
  return f;
}

// Impulse on a particle at velocity v from a static scene point (the depth camera's point
// cloud), FindAndHandleAugmentedRealityCollisionsUniformGridCell (RigidBodies/
// UniformGridDEM.cu:275-296): along the negated normal nn of the scene point, the scene at
// rest (rv = 0 - v), rp = scene point - particle, d = |rp| < contact tested by the caller.
__host__ __device__ __forceinline__ float3 scene_force(float3 rp, float dist, float3 vel,
                                                       float3 nn, float contact, float spring,
                                                       float damping, float shear,
                                                       float attraction) {
  const float3 nrm = ar::mk3(-nn.x, -nn.y, -nn.z);
  const float3 rv = ar::mk3(0.f - vel.x, 0.f - vel.y, 0.f - vel.z);
  const float3 tv = ar::sub(rv, ar::scl(ar::dot(rv, nrm), nrm));
  float3 f = ar::scl(-spring * (contact - dist), nrm);
  f = ar::add(f, ar::scl(damping, rv));
  f = ar::add(f, ar::scl(shear, tv));
  f = ar::add(f, ar::scl(attraction, rp));
  return f;
}

// collideStaticSpheresBVH (Kernels/RB_BVHKernels.cu:24-98): force on A from B plus the
// position correction it writes when the spheres overlap.
__device__ __forceinline__ float3 static_pair(float4 pa, float4 pb, float4 cm, float3 va,
                                              float3 vb, float ra, float rb,
                                              const ar_sim_params& p, float4* corr) {
  float3 rp = ar::mk3(pb.x - pa.x, pb.y - pa.y, pb.z - pa.z);
  float dist = sqrtf(ar::dot(rp, rp));
  float cd = ra + rb;
  if (!(dist < cd)) return ar::mk3(0.f, 0.f, 0.f);
  float3 f = spring_force(rp, dist, ar::sub(vb, va), cd, p.spring, p.damping, p.shear,
                          p.attraction);
  float3 nrm = ar::divs(rp, dist);
  float offset = -(cd - dist) / 2.f;
  float3 cb = ar::mk3(cm.x - pb.x, cm.y - pb.y, cm.z - pb.z);
  float3 ca = ar::mk3(cm.x - pa.x, cm.y - pa.y, cm.z - pa.z);
  if (sqrtf(ar::dot(cb, cb)) < sqrtf(ar::dot(ca, ca))) offset = -offset;
  *corr = make_float4(nrm.x * offset, nrm.y * offset, nrm.z * offset, 0.f);
  return f;
}

}  // namespace ar_dem
