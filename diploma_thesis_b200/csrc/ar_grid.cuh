// Uniform grid addressing: calcGridPos / calcGridHash (Kernels/particleKernels.cu:150-167,
// RigidBodies/UniformGridDEM.cu:25-41).
#pragma once
#include "ar_internal.cuh"

namespace ar_grid {

struct Grid {
  float ox, oy, oz;     // world origin
  float cx, cy, cz;     // cell edge per axis
  uint32_t gx, gy, gz;  // cells per axis (powers of two)

  static Grid from_params(const ar_sim_params& p) {
    Grid g;
    g.ox = p.world_origin[0]; g.oy = p.world_origin[1]; g.oz = p.world_origin[2];
    g.cx = p.cell_size[0]; g.cy = p.cell_size[1]; g.cz = p.cell_size[2];
    g.gx = p.grid_size[0]; g.gy = p.grid_size[1]; g.gz = p.grid_size[2];
    return g;
  }
  // cell = floor((p - origin) / cell) -- IEEE division, then floorf, then conversion to int
  __host__ __device__ __forceinline__ int3 cell_of(float3 p) const {
    return make_int3((int)floorf((p.x - ox) / cx), (int)floorf((p.y - oy) / cy),
                     (int)floorf((p.z - oz) / cz));
  }
  // wrap with & (G - 1), linearise z-major
  __host__ __device__ __forceinline__ uint32_t hash(int3 c) const {
    const uint32_t x = (uint32_t)c.x & (gx - 1), y = (uint32_t)c.y & (gy - 1),
                   z = (uint32_t)c.z & (gz - 1);
    return z * gy * gx + y * gx + x;
  }
};

}  // namespace ar_grid
