// (f) Depth-camera ingestion for the static scene: a 16-bit depth image -> the static point
// cloud (world positions, radii, and the 5-float vertex records the renderer's buffer takes),
// then per-pixel normals from the 8-neighbourhood.  Restates RGBDloader and computeNormals
// (Kernels/customRangeImageLoader.cu:14-113, 122-177), the kernels loadRangeImage launches
// (:179-221); the GL buffer the reference maps for the vertex records is a plain device buffer
// here, and the image is read by the caller (the reference uses OpenCV,
// Particles/loadRangeDataFromFile.cpp:150-200).
//
// Arithmetic in the reference's order: the hard-coded intrinsics (focal 517.3 / 516.5, centre
// 318.6 / 255.3, depth / 5000, "no depth" below 0.01 -> z = -1000), the camera matrix
// transposed and applied to (x, y, z, 0), the hard-coded gravity rotation built from the
// normalised accelerometer vector, glm 0.9.7's matrix-vector pairing ((m0 v0 + m1 v1) +
// (m2 v2 + m3 v3)), then (x, -y, -z).  Normals: normalize(cross(p(y+1) - p(y-1), p(x+1) -
// p(x-1))), with the inverse length as 1 / sqrtf (IEEE; the reference's device build takes
// helper_math's rsqrtf, its host build 1 / sqrtf), border pixels left untouched.  The
// reference skips pixels whose index exceeds (width - 1) * (height - 1), and so does this; its
// launch covers only whole 16 x 32 blocks, this one every pixel.
#include "ar_internal.cuh"

namespace {

struct Mat4 {
  float c[4][4];  // column-major, c[column][row] (the glm::mat4 layout)
};

// glm 0.9.7 mat4 * vec4: per component (m0 v0 + m1 v1) + (m2 v2 + m3 v3)
__device__ __forceinline__ float4 mat4_mul(const Mat4& m, float4 v) {
  float r[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float a0 = m.c[0][i] * v.x + m.c[1][i] * v.y;
    const float a1 = m.c[2][i] * v.z + m.c[3][i] * v.w;
    r[i] = a0 + a1;
  }
  return make_float4(r[0], r[1], r[2], r[3]);
}

__global__ void __launch_bounds__(512) range_cloud_kernel(const uint16_t* __restrict__ depth,
                                                          int w, int h, Mat4 cam_t,
                                                          float radius,
                                                          float4* __restrict__ pos4,
                                                          float* __restrict__ radii,
                                                          float* __restrict__ vao5) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= w || y >= h) return;
  const long index = (long)y * w + x;
  if (index > (long)(w - 1) * (h - 1)) return;
  const float fx = (float)517.3, fy = (float)516.5, cx = (float)318.6, cy = (float)255.3;
  float pz = (float)__ldg(depth + index);
  pz /= 5000.f;
  radii[index] = radius;
  if ((double)pz < 0.01) pz = -1000.f;
  const float px = pz * ((float)x - cx) / fx;
  const float py = pz * ((float)y - cy) / fy;
  float4 t = mat4_mul(cam_t, make_float4(px, py, pz, 0.f));
  // the accelerometer vector, normalised as glm does (v * (1 / sqrt(dot(v, v))))
  const float gx0 = (float)0.478957, gy0 = (float)-8.010560, gz0 = (float)4.166928;
  const float inv = 1.0f / sqrtf(gx0 * gx0 + gy0 * gy0 + gz0 * gz0);
  const float gx = gx0 * inv, gy = gy0 * inv, gz = gz0 * inv;
  Mat4 grav;
  const float cols[16] = {1.f, 0.f, 0.f, 0.f, -gx, -gy, -gz, 0.f,
                          0.f, gz, -gy, 0.f, 0.f, 0.f, 0.f, 1.f};
#pragma unroll
  for (int i = 0; i < 16; ++i) grav.c[i / 4][i % 4] = cols[i];
  t = mat4_mul(grav, t);
  const float ox = t.x, oy = -t.y, oz = -t.z;
  if (vao5) {
    float* v = vao5 + 5 * index;
    v[0] = ox;
    v[1] = oy;
    v[2] = oz;
    v[3] = (float)x / (float)w;
    v[4] = (float)y / (float)h;
  }
  pos4[index] = make_float4(ox, oy, oz, 0.f);
}

__global__ void __launch_bounds__(512) range_normals_kernel(const float4* __restrict__ pos4,
                                                            int w, int h,
                                                            float4* __restrict__ norm4) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x > w - 2 || x == 0 || y == 0 || y > h - 2) return;
  const float4 up = __ldg(pos4 + (long)(y - 1) * w + x), right = __ldg(pos4 + (long)y * w + x + 1);
  const float4 down = __ldg(pos4 + (long)(y + 1) * w + x), left = __ldg(pos4 + (long)y * w + x - 1);
  const float3 dx = ar::mk3(right.x - left.x, right.y - left.y, right.z - left.z);
  const float3 dy = ar::mk3(down.x - up.x, down.y - up.y, down.z - up.z);
  const float3 c = ar::mk3(dy.y * dx.z - dy.z * dx.y, dy.z * dx.x - dy.x * dx.z,
                           dy.x * dx.y - dy.y * dx.x);
  const float inv = 1.0f / sqrtf(c.x * c.x + c.y * c.y + c.z * c.z);
  norm4[(long)y * w + x] = make_float4(c.x * inv, c.y * inv, c.z * inv, 0.f);
}

constexpr int kRangeBlockX = 16, kRangeBlockY = 32;  // the reference's block shape

bool bad_image(int w, int h) { return w < 1 || h < 1 || (long)w * h >= (1l << 31); }

}  // namespace

extern "C" {

ar_status ar_range_image_cloud(ar_ctx* ctx, const uint16_t* depth, int width, int height,
                               const float* camera16, float particle_radius, float* static_pos4,
                               float* static_radii, float* vao5, ar_stream_t stream) {
  if (!ctx || !depth || !camera16 || !static_pos4 || !static_radii || bad_image(width, height))
    return AR_ERR_INVALID_ARG;
  if (((uintptr_t)static_pos4 & 15u) != 0) {
    arh::set_error("ar_range_image_cloud: static_pos4 must be 16-byte aligned");
    return AR_ERR_INVALID_ARG;
  }
  Mat4 t;  // the camera matrix transposed (the reference transposes it in the kernel)
  for (int c = 0; c < 4; ++c)
    for (int r = 0; r < 4; ++r) t.c[c][r] = camera16[4 * r + c];
  const dim3 block(kRangeBlockX, kRangeBlockY);
  const dim3 grid((unsigned)((width + kRangeBlockX - 1) / kRangeBlockX),
                  (unsigned)((height + kRangeBlockY - 1) / kRangeBlockY));
  range_cloud_kernel<<<grid, block, 0, arh::stream(stream)>>>(
      depth, width, height, t, particle_radius, (float4*)static_pos4, static_radii, vao5);
  return arh::check_launch("ar_range_image_cloud");
}

ar_status ar_range_image_normals(ar_ctx* ctx, const float* static_pos4, int width, int height,
                                 float* static_norm4, ar_stream_t stream) {
  if (!ctx || !static_pos4 || !static_norm4 || bad_image(width, height))
    return AR_ERR_INVALID_ARG;
  if ((((uintptr_t)static_pos4 | (uintptr_t)static_norm4) & 15u) != 0) {
    arh::set_error("ar_range_image_normals: pointers must be 16-byte aligned");
    return AR_ERR_INVALID_ARG;
  }
  const dim3 block(kRangeBlockX, kRangeBlockY);
  const dim3 grid((unsigned)((width + kRangeBlockX - 1) / kRangeBlockX),
                  (unsigned)((height + kRangeBlockY - 1) / kRangeBlockY));
  range_normals_kernel<<<grid, block, 0, arh::stream(stream)>>>(
      (const float4*)static_pos4, width, height, (float4*)static_norm4);
  return arh::check_launch("ar_range_image_normals");
}

}  // extern "C"
