// glm 0.9.7 operations used by the reference kernels, restated with the same evaluation
// order (Libs/glm/glm/detail/type_mat3x3.inl:501-548, gtc/quaternion.inl:42-49,263-273,
// 384-397,598-623).  Matrices are glm::mat3 memory: column-major, m[c*3 + r].
// Quaternions are glm::quat memory order (x, y, z, w).
#pragma once
#include "ar_internal.cuh"

namespace ar_glm {

// glm vec3 dot: (x + y) + z
__host__ __device__ __forceinline__ float dot3(float3 a, float3 b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
// glm::cross
__host__ __device__ __forceinline__ float3 cross3(float3 x, float3 y) {
  return ar::mk3(x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y);
}
// mat3 * vec3 (type_mat3x3.inl:501-507)
__host__ __device__ __forceinline__ float3 mv(const float* m, float3 v) {
  return ar::mk3(m[0] * v.x + m[3] * v.y + m[6] * v.z, m[1] * v.x + m[4] * v.y + m[7] * v.z,
                 m[2] * v.x + m[5] * v.y + m[8] * v.z);
}
// mat3 * mat3 (type_mat3x3.inl:519-548)
__host__ __device__ __forceinline__ void mm(const float* a, const float* b, float* r) {
  for (int c = 0; c < 3; ++c)
    for (int rr = 0; rr < 3; ++rr)
      r[c * 3 + rr] = a[0 * 3 + rr] * b[c * 3 + 0] + a[1 * 3 + rr] * b[c * 3 + 1] +
                      a[2 * 3 + rr] * b[c * 3 + 2];
}
__host__ __device__ __forceinline__ void transpose(const float* a, float* t) {
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) t[c * 3 + r] = a[r * 3 + c];
}
// mat3_cast (gtc/quaternion.inl:598-623)
__host__ __device__ __forceinline__ void mat3_cast(float4 q, float* m) {
  float qxx = q.x * q.x, qyy = q.y * q.y, qzz = q.z * q.z;
  float qxz = q.x * q.z, qxy = q.x * q.y, qyz = q.y * q.z;
  float qwx = q.w * q.x, qwy = q.w * q.y, qwz = q.w * q.z;
  m[0] = 1 - 2 * (qyy + qzz);
  m[1] = 2 * (qxy + qwz);
  m[2] = 2 * (qxz - qwy);
  m[3] = 2 * (qxy - qwz);
  m[4] = 1 - 2 * (qxx + qzz);
  m[5] = 2 * (qyz + qwx);
  m[6] = 2 * (qxz + qwy);
  m[7] = 2 * (qyz - qwx);
  m[8] = 1 - 2 * (qxx + qyy);
}
// quat normalize (gtc/quaternion.inl:384-397): dot = (xx + yy) + (zz + ww)
__host__ __device__ __forceinline__ float4 qnormalize(float4 q) {
  float len = sqrtf((q.x * q.x + q.y * q.y) + (q.z * q.z + q.w * q.w));
  if (len <= 0.f) return make_float4(0.f, 0.f, 0.f, 1.f);
  float inv = 1.f / len;
  return make_float4(q.x * inv, q.y * inv, q.z * inv, q.w * inv);
}
// quat product p * q (gtc/quaternion.inl:263-273)
__host__ __device__ __forceinline__ float4 qmul(float4 p, float4 q) {
  float4 r;
  r.w = p.w * q.w - p.x * q.x - p.y * q.y - p.z * q.z;
  r.x = p.w * q.x + p.x * q.w + p.y * q.z - p.z * q.y;
  r.y = p.w * q.y + p.y * q.w + p.z * q.x - p.x * q.z;
  r.z = p.w * q.z + p.z * q.w + p.x * q.y - p.y * q.x;
  return r;
}
// mat4_cast(q) * vec4(v, 0) (type_mat4x4.inl:610-650): ((m0 x + m1 y) + (m2 z + 0 * 0))
__host__ __device__ __forceinline__ float3 rotate_mat4(const float* m, float3 v) {
  return ar::mk3((m[0] * v.x + m[3] * v.y) + (m[6] * v.z + 0.f * 0.f),
                 (m[1] * v.x + m[4] * v.y) + (m[7] * v.z + 0.f * 0.f),
                 (m[2] * v.x + m[5] * v.y) + (m[8] * v.z + 0.f * 0.f));
}

}  // namespace ar_glm
