// (a13) grid hash, (a14) reorder + cell ranges, (a15) DEM gather, grid contact pairs.
// Stage entry points with the reference wrappers' semantics; the fused step uses its own
// kernels (ar_pipeline.cu) built from the same device functions.
#include <cstring>

#include "ar_internal.cuh"
#include "ar_dem.cuh"
#include "ar_grid.cuh"

namespace {

__global__ void __launch_bounds__(256) calc_hash_kernel(ar_grid::Grid g,
                                                        const float4* __restrict__ pos, int n,
                                                        uint32_t* __restrict__ hash,
                                                        uint32_t* __restrict__ idx) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 p = __ldg(pos + i);
    hash[i] = g.hash(g.cell_of(ar::xyz(p)));
    if (idx) idx[i] = (uint32_t)i;
  }
}

__global__ void __launch_bounds__(256) fill_kernel(uint32_t* __restrict__ a, long n, uint32_t v) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    a[i] = v;
}

// reorderDataAndFindCellStartD (Kernels/particleKernels.cu:193-258): the previous slot's hash
// comes straight from global memory (cached) instead of a shared-memory halo.
__global__ void __launch_bounds__(256) reorder_kernel(const uint32_t* __restrict__ hash,
                                                      const uint32_t* __restrict__ idx,
                                                      const float4* __restrict__ pos,
                                                      const float4* __restrict__ vel, int n,
                                                      uint32_t* __restrict__ cell_start,
                                                      uint32_t* __restrict__ cell_end,
                                                      float4* __restrict__ sorted_pos,
                                                      float4* __restrict__ sorted_vel) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t h = __ldg(hash + i);
    if (i == 0 || h != __ldg(hash + i - 1)) {
      cell_start[h] = i;
      if (i > 0) cell_end[__ldg(hash + i - 1)] = i;
    }
    if (i == n - 1) cell_end[h] = i + 1;
    const uint32_t s = __ldg(idx + i);
    sorted_pos[i] = __ldg(pos + s);
    if (sorted_vel) sorted_vel[i] = __ldg(vel + s);
  }
}

// FindAndHandleRigidBodyCollisionsUniformGridKernel (RigidBodies/UniformGridDEM.cu:133-204).
__global__ void __launch_bounds__(128) collide_grid_kernel(
    ar_sim_params prm, ar_grid::Grid g, const int32_t* __restrict__ rb_idx,
    const float4* __restrict__ spos, const float4* __restrict__ svel,
    const float4* __restrict__ rel, const uint32_t* __restrict__ gidx,
    const uint32_t* __restrict__ cstart, const uint32_t* __restrict__ cend, int n,
    float4* __restrict__ p_force, float4* __restrict__ p_torque) {
  const int index = blockIdx.x * blockDim.x + threadIdx.x;
  if (index >= n) return;
  const float3 pos = ar::xyz(__ldg(spos + index));
  const float3 vel = ar::xyz(__ldg(svel + index));
  const int3 gp = g.cell_of(pos);
  const uint32_t orig = __ldg(gidx + index);
  const int body = __ldg(rb_idx + orig);
  const float thr = 2.0f * prm.particle_radius;
  float3 lin = ar::mk3(0.f, 0.f, 0.f);
  for (int z = -1; z <= 1; ++z)
    for (int y = -1; y <= 1; ++y)
      for (int x = -1; x <= 1; ++x) {
        float3 cell_f = ar::mk3(0.f, 0.f, 0.f);
        const uint32_t h = g.hash(make_int3(gp.x + x, gp.y + y, gp.z + z));
        const uint32_t st = __ldg(cstart + h);
        if (st != ar::kEmpty) {
          const uint32_t en = __ldg(cend + h);
          for (uint32_t j = st; j < en; ++j) {
            const int b2 = __ldg(rb_idx + __ldg(gidx + j));
            if (j == (uint32_t)index || body == b2) continue;
            const float3 p2 = ar::xyz(__ldg(spos + j));
            const float3 rp = ar::sub(p2, pos);
            const float dist = sqrtf(ar::dot(rp, rp));
            if (dist < thr) {
              const float3 v2 = ar::xyz(__ldg(svel + j));
              cell_f = ar::add(cell_f, ar_dem::spring_force(rp, dist, ar::sub(v2, vel), thr,
                                                            prm.spring, prm.damping, prm.shear,
                                                            prm.attraction));
            }
          }
        }
        lin = ar::add(lin, cell_f);
      }
  float4 f = p_force[orig];
  p_force[orig] = make_float4(f.x + lin.x, f.y + lin.y, f.z + lin.z, f.w + 0.f);
  const float3 t = ar::cross(ar::xyz(__ldg(rel + orig)), lin);
  float4 q = p_torque[orig];
  p_torque[orig] = make_float4(q.x + t.x, q.y + t.y, q.z + t.z, q.w + 0.f);
}

// FindAndHandleAugmentedRealityCollisionsUniformGridKernel (RigidBodies/UniformGridDEM.cu:
// 243-377): per sorted particle, the static scene's particles (sorted into the same grid, with
// their own cell table) in the 27 neighbour cells, z, y, x order; for d < 2r a DEM impulse
// along the negated scene normal of the scene particle (unsorted normals, indexed through the
// scene's sorted indices): -spring (2r - d) n + damping v_rel + shear v_t + attraction p_rel,
// v_rel = 0 - v.  Summed per cell, then added to the particle's linear impulse, and
// rel x sum to its angular impulse; colour set to green on any contact.
__global__ void __launch_bounds__(128) collide_static_kernel(
    ar_sim_params prm, ar_grid::Grid g, const float4* __restrict__ spos,
    const float4* __restrict__ svel, const float4* __restrict__ rel,
    const float4* __restrict__ scene_spos, const float4* __restrict__ scene_normals,
    const uint32_t* __restrict__ gidx, const uint32_t* __restrict__ scene_gidx,
    const uint32_t* __restrict__ cstart, const uint32_t* __restrict__ cend, int n,
    float4* __restrict__ p_lin, float4* __restrict__ p_ang, float4* __restrict__ color) {
  const int index = blockIdx.x * blockDim.x + threadIdx.x;
  if (index >= n) return;
  const float3 pos = ar::xyz(__ldg(spos + index));
  const float3 vel = ar::xyz(__ldg(svel + index));
  const int3 gp = g.cell_of(pos);
  const uint32_t orig = __ldg(gidx + index);
  const float thr = 2.0f * prm.particle_radius;
  int contacts = 0;
  float4 lin = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int z = -1; z <= 1; ++z)
    for (int y = -1; y <= 1; ++y)
      for (int x = -1; x <= 1; ++x) {
        float4 cell_f = make_float4(0.f, 0.f, 0.f, 0.f);
        const uint32_t h = g.hash(make_int3(gp.x + x, gp.y + y, gp.z + z));
        const uint32_t st = __ldg(cstart + h);
        if (st != ar::kEmpty) {
          const uint32_t en = __ldg(cend + h);
          for (uint32_t j = st; j < en; ++j) {
            const uint32_t o2 = __ldg(scene_gidx + j);
            const float3 rp = ar::sub(ar::xyz(__ldg(scene_spos + j)), pos);
            const float dist = sqrtf(ar::dot(rp, rp));
            if (!(dist < thr)) continue;
            const float3 f = ar_dem::scene_force(rp, dist, vel, ar::xyz(__ldg(scene_normals + o2)),
                                                 thr, prm.spring, prm.damping, prm.shear,
                                                 prm.attraction);
            cell_f = make_float4(cell_f.x + f.x, cell_f.y + f.y, cell_f.z + f.z, cell_f.w + 0.f);
            ++contacts;
          }
        }
        lin = make_float4(lin.x + cell_f.x, lin.y + cell_f.y, lin.z + cell_f.z, lin.w + cell_f.w);
      }
  if (contacts && color) color[orig] = make_float4(0.f, 1.f, 0.f, 0.f);
  const float4 a = p_lin[orig];
  p_lin[orig] = make_float4(a.x + lin.x, a.y + lin.y, a.z + lin.z, a.w + lin.w);
  const float3 t = ar::cross(ar::xyz(__ldg(rel + orig)), ar::xyz(lin));
  const float4 b = p_ang[orig];
  p_ang[orig] = make_float4(b.x + t.x, b.y + t.y, b.z + t.z, b.w + 0.f);
}

// collideD / collideCell / collideSpheres (Kernels/particleKernels.cu:261-406): the particle
// variant -- every occupant that passes the body test contributes (zero when apart), torque
// accumulates per cell, free particles (body -1) get their velocity updated instead.
__global__ void __launch_bounds__(128) collide_particles_kernel(
    ar_sim_params prm, ar_grid::Grid g, const int32_t* __restrict__ rb_idx,
    const float4* __restrict__ spos, const float4* __restrict__ svel,
    const float4* __restrict__ rel, const uint32_t* __restrict__ gidx,
    const uint32_t* __restrict__ cstart, const uint32_t* __restrict__ cend, int n,
    float4* __restrict__ p_force, float4* __restrict__ p_torque, float4* __restrict__ new_vel) {
  const int index = blockIdx.x * blockDim.x + threadIdx.x;
  if (index >= n) return;
  const float3 pos = ar::xyz(__ldg(spos + index));
  const float3 vel = ar::xyz(__ldg(svel + index));
  const int3 gp = g.cell_of(pos);
  const uint32_t orig = __ldg(gidx + index);
  const int body = __ldg(rb_idx + orig);
  const float cd = prm.particle_radius + prm.particle_radius;
  const float3 r3 = ar::xyz(__ldg(rel + orig));
  float3 force = ar::mk3(0.f, 0.f, 0.f), torque = ar::mk3(0.f, 0.f, 0.f);
  for (int z = -1; z <= 1; ++z)
    for (int y = -1; y <= 1; ++y)
      for (int x = -1; x <= 1; ++x) {
        float3 cf = ar::mk3(0.f, 0.f, 0.f);
        const uint32_t h = g.hash(make_int3(gp.x + x, gp.y + y, gp.z + z));
        const uint32_t st = __ldg(cstart + h);
        if (st != ar::kEmpty) {
          const uint32_t en = __ldg(cend + h);
          for (uint32_t j = st; j < en; ++j) {
            if (!(j != (uint32_t)index && (body != __ldg(rb_idx + __ldg(gidx + j)) || body == -1)))
              continue;
            const float3 p2 = ar::xyz(__ldg(spos + j));
            const float3 rp = ar::sub(p2, pos);
            const float dist = sqrtf(ar::dot(rp, rp));
            float3 f = ar::mk3(0.f, 0.f, 0.f);
            if (dist < cd)
              f = ar_dem::spring_force(rp, dist, ar::sub(ar::xyz(__ldg(svel + j)), vel), cd,
                                       prm.spring, prm.damping, prm.shear, prm.attraction);
            cf = ar::add(cf, f);
          }
        }
        force = ar::add(force, cf);
        torque = ar::add(torque, ar::cross(r3, cf));
      }
  if (body == -1) {
    if (new_vel) new_vel[orig] = make_float4(vel.x + force.x, vel.y + force.y, vel.z + force.z, 0.f);
  } else {
    p_force[orig] = make_float4(force.x, force.y, force.z, 0.f);
    p_torque[orig] = make_float4(torque.x, torque.y, torque.z, 0.f);
  }
}

__global__ void __launch_bounds__(128) pairs_grid_kernel(
    float two_r, ar_grid::Grid g, const int32_t* __restrict__ rb_idx,
    const float4* __restrict__ spos, const uint32_t* __restrict__ gidx,
    const uint32_t* __restrict__ cstart, const uint32_t* __restrict__ cend, int n,
    int2* __restrict__ pairs, int capacity, int* __restrict__ count, int* __restrict__ err) {
  const int index = blockIdx.x * blockDim.x + threadIdx.x;
  if (index >= n) return;
  const float3 pos = ar::xyz(__ldg(spos + index));
  const int3 gp = g.cell_of(pos);
  const uint32_t orig = __ldg(gidx + index);
  const int body = __ldg(rb_idx + orig);
  for (int z = -1; z <= 1; ++z)
    for (int y = -1; y <= 1; ++y)
      for (int x = -1; x <= 1; ++x) {
        const uint32_t h = g.hash(make_int3(gp.x + x, gp.y + y, gp.z + z));
        const uint32_t st = __ldg(cstart + h);
        if (st == ar::kEmpty) continue;
        const uint32_t en = __ldg(cend + h);
        for (uint32_t j = st; j < en; ++j) {
          if (j <= (uint32_t)index) continue;  // each unordered pair from its lower slot
          const uint32_t o2 = __ldg(gidx + j);
          if (__ldg(rb_idx + o2) == body) continue;
          if (!ar_dem::touching(pos, ar::xyz(__ldg(spos + j)), two_r)) continue;
          int slot = atomicAdd(count, 1);
          if (slot < capacity)
            pairs[slot] = make_int2(min((int)orig, (int)o2), max((int)orig, (int)o2));
          else
            ar::raise_error(err, ar::kErrOverflow);
        }
      }
}

bool pow2(uint32_t v) { return v && !(v & (v - 1)); }

ar_status grid_from_params(const ar_sim_params* p, ar_grid::Grid* g) {
  for (int a = 0; a < 3; ++a)
    if (!pow2(p->grid_size[a])) {
      arh::set_error("grid_size must be powers of two (the hash wraps with & (G-1))");
      return AR_ERR_INVALID_ARG;
    }
  *g = ar_grid::Grid::from_params(*p);
  return AR_OK;
}

}  // namespace

extern "C" {

ar_status ar_calc_hash(ar_ctx* ctx, const ar_sim_params* params, const float* pos4, int n,
                       uint32_t* hash, uint32_t* idx, ar_stream_t stream) {
  if (!ctx || !params || n < 0 || (n > 0 && (!pos4 || !hash))) return AR_ERR_INVALID_ARG;
  ar_grid::Grid g;
  ar_status s = grid_from_params(params, &g);
  if (s != AR_OK || n == 0) return s;
  unsigned grid = arh::grid_for(n, 256);
  if (grid > (unsigned)ctx->num_sms * 8) grid = ctx->num_sms * 8;
  calc_hash_kernel<<<grid, 256, 0, arh::stream(stream)>>>(g, (const float4*)pos4, n, hash, idx);
  return arh::check_launch("ar_calc_hash");
}

ar_status ar_reorder_cells(ar_ctx* ctx, const uint32_t* sorted_hash, const uint32_t* sorted_idx,
                           const float* pos4, const float* vel4, int n, uint32_t num_cells,
                           uint32_t* cell_start, uint32_t* cell_end, float* sorted_pos4,
                           float* sorted_vel4, ar_stream_t stream) {
  if (!ctx || n < 0 || !cell_start || !cell_end ||
      (n > 0 && (!sorted_hash || !sorted_idx || !pos4 || !sorted_pos4 ||
                 (sorted_vel4 && !vel4))))
    return AR_ERR_INVALID_ARG;
  cudaStream_t st = arh::stream(stream);
  unsigned cap = (unsigned)ctx->num_sms * 8;
  unsigned g1 = arh::grid_for(num_cells, 256);
  fill_kernel<<<g1 > cap ? cap : g1, 256, 0, st>>>(cell_start, num_cells, ar::kEmpty);
  if (n > 0) {
    unsigned g2 = arh::grid_for(n, 256);
    reorder_kernel<<<g2 > cap ? cap : g2, 256, 0, st>>>(
        sorted_hash, sorted_idx, (const float4*)pos4, (const float4*)vel4, n, cell_start,
        cell_end, (float4*)sorted_pos4, (float4*)sorted_vel4);
  }
  return arh::check_launch("ar_reorder_cells");
}

ar_status ar_collide_grid_dem(ar_ctx* ctx, const ar_sim_params* params, const int32_t* rb_idx,
                              const float* sorted_pos4, const float* sorted_vel4,
                              const float* rel4, const uint32_t* grid_idx,
                              const uint32_t* cell_start, const uint32_t* cell_end, int n,
                              float* p_force4, float* p_torque4, ar_stream_t stream) {
  if (!ctx || !params || n < 0 ||
      (n > 0 && (!rb_idx || !sorted_pos4 || !sorted_vel4 || !rel4 || !grid_idx || !cell_start ||
                 !cell_end || !p_force4 || !p_torque4)))
    return AR_ERR_INVALID_ARG;
  ar_grid::Grid g;
  ar_status s = grid_from_params(params, &g);
  if (s != AR_OK || n == 0) return s;
  collide_grid_kernel<<<arh::grid_for(n, 128), 128, 0, arh::stream(stream)>>>(
      *params, g, rb_idx, (const float4*)sorted_pos4, (const float4*)sorted_vel4,
      (const float4*)rel4, grid_idx, cell_start, cell_end, n, (float4*)p_force4,
      (float4*)p_torque4);
  return arh::check_launch("ar_collide_grid_dem");
}

ar_status ar_collide_static_scene_dem(ar_ctx* ctx, const ar_sim_params* params,
                                      const float* sorted_pos4, const float* sorted_vel4,
                                      const float* rel4, const float* scene_sorted_pos4,
                                      const float* scene_normals4, const uint32_t* grid_idx,
                                      const uint32_t* scene_grid_idx,
                                      const uint32_t* scene_cell_start,
                                      const uint32_t* scene_cell_end, int n,
                                      float* p_linear4, float* p_angular4, float* color4,
                                      ar_stream_t stream) {
  if (!ctx || !params || n < 0 ||
      (n > 0 && (!sorted_pos4 || !sorted_vel4 || !rel4 || !scene_sorted_pos4 ||
                 !scene_normals4 || !grid_idx || !scene_grid_idx || !scene_cell_start ||
                 !scene_cell_end || !p_linear4 || !p_angular4)))
    return AR_ERR_INVALID_ARG;
  ar_grid::Grid g;
  ar_status s = grid_from_params(params, &g);
  if (s != AR_OK || n == 0) return s;
  collide_static_kernel<<<arh::grid_for(n, 128), 128, 0, arh::stream(stream)>>>(
      *params, g, (const float4*)sorted_pos4, (const float4*)sorted_vel4, (const float4*)rel4,
      (const float4*)scene_sorted_pos4, (const float4*)scene_normals4, grid_idx, scene_grid_idx,
      scene_cell_start, scene_cell_end, n, (float4*)p_linear4, (float4*)p_angular4,
      (float4*)color4);
  return arh::check_launch("ar_collide_static_scene_dem");
}

ar_status ar_collide_grid_particles(ar_ctx* ctx, const ar_sim_params* params,
                                    const int32_t* rb_idx, const float* sorted_pos4,
                                    const float* sorted_vel4, const float* rel4,
                                    const uint32_t* grid_idx, const uint32_t* cell_start,
                                    const uint32_t* cell_end, int n, float* p_force4,
                                    float* p_torque4, float* new_vel4, ar_stream_t stream) {
  if (!ctx || !params || n < 0 ||
      (n > 0 && (!rb_idx || !sorted_pos4 || !sorted_vel4 || !rel4 || !grid_idx || !cell_start ||
                 !cell_end || !p_force4 || !p_torque4)))
    return AR_ERR_INVALID_ARG;
  ar_grid::Grid g;
  ar_status s = grid_from_params(params, &g);
  if (s != AR_OK || n == 0) return s;
  collide_particles_kernel<<<arh::grid_for(n, 128), 128, 0, arh::stream(stream)>>>(
      *params, g, rb_idx, (const float4*)sorted_pos4, (const float4*)sorted_vel4,
      (const float4*)rel4, grid_idx, cell_start, cell_end, n, (float4*)p_force4,
      (float4*)p_torque4, (float4*)new_vel4);
  return arh::check_launch("ar_collide_grid_particles");
}

ar_status ar_fill_f32(ar_ctx* ctx, float* dst, long n, float value, ar_stream_t stream) {
  if (!ctx || n < 0 || (n > 0 && !dst)) return AR_ERR_INVALID_ARG;
  if (n == 0) return AR_OK;
  uint32_t bits;
  memcpy(&bits, &value, 4);
  unsigned g = arh::grid_for(n, 256);
  unsigned cap = (unsigned)ctx->num_sms * 8;
  fill_kernel<<<g > cap ? cap : g, 256, 0, arh::stream(stream)>>>((uint32_t*)dst, n, bits);
  return arh::check_launch("ar_fill_f32");
}

ar_status ar_pairs_grid(ar_ctx* ctx, const ar_sim_params* params, const int32_t* rb_idx,
                        const float* sorted_pos4, const uint32_t* grid_idx,
                        const uint32_t* cell_start, const uint32_t* cell_end, int n,
                        int32_t* pairs2, int capacity, int32_t* d_count, ar_stream_t stream) {
  if (!ctx || !params || n < 0 || capacity < 0 || !d_count ||
      (n > 0 && (!rb_idx || !sorted_pos4 || !grid_idx || !cell_start || !cell_end ||
                 (capacity > 0 && !pairs2))))
    return AR_ERR_INVALID_ARG;
  ar_grid::Grid g;
  ar_status s = grid_from_params(params, &g);
  if (s != AR_OK) return s;
  cudaStream_t st = arh::stream(stream);
  cudaMemsetAsync(d_count, 0, sizeof(int32_t), st);
  if (n == 0) return arh::check_launch("ar_pairs_grid");
  pairs_grid_kernel<<<arh::grid_for(n, 128), 128, 0, st>>>(
      2.0f * params->particle_radius, g, rb_idx, (const float4*)sorted_pos4, grid_idx,
      cell_start, cell_end, n, (int2*)pairs2, capacity, d_count, ctx->d_err);
  return arh::check_launch("ar_pairs_grid");
}

}  // extern "C"
