// (f) Rigid bodies against a static scene (the augmented-reality point cloud): the impulse
// variant of the collision, the deepest-contact search and the contact gather of the
// sequential-impulse path.  The scene is a point cloud with normals, sorted into its own
// uniform grid (scene_cell_start / scene_cell_end, scene_sorted_pos4 in cell order,
// scene_grid_idx the cloud index of each sorted point).
#include <algorithm>

#include "ar_glm.cuh"
#include "ar_grid.cuh"
#include "ar_internal.cuh"

namespace {

// collideARSpheresBaraffExact (Kernels/RB_UniformGridKernels.cu:420-466): an impulse along
// the line of centres at the exact contact point, restitution params.ARrestitution, applied
// to a body with inverse inertia `inertia` (glm::mat3 layout) and mass `mass`; the torque arm
// is the contact point minus the body centre (particle position minus its offset).
__device__ __forceinline__ void baraff_exact(float3 pa, float3 pb, float3 va, float ra, float rb,
                                             const float* inertia, float3 rel, float mass,
                                             float restitution, int* ncol, float3* lf,
                                             float3* lt) {
  const float3 rp = ar::sub(pa, pb);
  const float dist = sqrtf(ar::dot(rp, rp));
  const float cd = ra + rb;
  if (!(dist < cd)) return;
  ++*ncol;
  const float t = ra / (ra + rb);
  const float3 d = ar::sub(pb, pa);
  const float3 cp = ar::add(pa, ar::mk3(t * d.x, t * d.y, t * d.z));
  const float3 nrm = ar::divs(rp, dist);
  const float rv = ar::dot(va, nrm);
  const float3 cm = ar::sub(pa, rel);
  const float3 ra3 = ar::mk3(cp.x - cm.x, cp.y - cm.y, cp.z - cm.z);
  const float denom =
      ar_glm::dot3(ar_glm::cross3(ar_glm::mv(inertia, ar_glm::cross3(ra3, nrm)), ra3), nrm) +
      1.f / mass;
  const float j = -(1 + restitution) * rv / denom;
  const float3 f = ar::mk3(nrm.x * j, nrm.y * j, nrm.z * j);
  *lf = ar::add(*lf, f);
  *lt = ar::add(*lt, ar::cross(ra3, f));
}

// ARcollisionsUniformGridKernel with ARCellRigidBody (Kernels/RB_UniformGridKernels.cu:
// 513-667).  As the reference does, every one of the 27 iterations of the neighbour loop
// examines the particle's own cell (it passes gridPos, not neighbourPos, :613), and each
// iteration's partial force and torque are added to the totals.  A particle of a body gets
// its force, torque and collision count written at its original index; a free particle
// (body index -1) gets the force added to its velocity instead, computed with a zero inverse
// inertia and unit mass (the reference reads the body arrays at index -1 there).
__global__ void __launch_bounds__(128) static_impulse_kernel(
    ar_sim_params prm, ar_grid::Grid g, const int32_t* __restrict__ rb_idx,
    const float4* __restrict__ rel4, const float* __restrict__ inertia9,
    const float* __restrict__ mass, const float* __restrict__ scene_radii,
    const float4* __restrict__ spos, const float4* __restrict__ svel,
    const float4* __restrict__ scene_spos, const uint32_t* __restrict__ gidx,
    const uint32_t* __restrict__ scene_gidx, const uint32_t* __restrict__ cstart,
    const uint32_t* __restrict__ cend, int n, float4* __restrict__ p_force,
    float4* __restrict__ p_torque, int32_t* __restrict__ p_count, float4* __restrict__ new_vel,
    float4* __restrict__ color) {
  for (int index = blockIdx.x * blockDim.x + threadIdx.x; index < n;
       index += gridDim.x * blockDim.x) {
    const float3 pos = ar::xyz(__ldg(spos + index));
    const float3 vel = ar::xyz(__ldg(svel + index));
    const int3 gp = g.cell_of(pos);
    const uint32_t orig = __ldg(gidx + index);
    const int b = __ldg(rb_idx + orig);
    float ib[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    float m = 1.f;
    if (b >= 0) {
      for (int k = 0; k < 9; ++k) ib[k] = __ldg(inertia9 + 9 * (size_t)b + k);
      m = __ldg(mass + b);
    }
    const float3 rel = ar::xyz(__ldg(rel4 + orig));
    float3 force = ar::mk3(0.f, 0.f, 0.f), torque = force;
    int ncol = 0;
    const uint32_t h = g.hash(gp);  // the cell every iteration examines
    const uint32_t st = __ldg(cstart + h);
    for (int it = 0; it < 27; ++it) {
      float3 lf = ar::mk3(0.f, 0.f, 0.f), lt = lf;
      if (st != ar::kEmpty) {
        const uint32_t en = __ldg(cend + h);
        for (uint32_t j = st; j < en; ++j) {
          const uint32_t o2 = __ldg(scene_gidx + j);
          baraff_exact(pos, ar::xyz(__ldg(scene_spos + j)), vel, prm.particle_radius,
                       __ldg(scene_radii + o2), ib, rel, m, prm.ar_restitution, &ncol, &lf, &lt);
        }
      }
      force = ar::add(force, lf);
      torque = ar::add(torque, lt);
    }
    if (ncol && color) color[orig] = make_float4(0.f, 1.f, 0.f, 0.f);
    if (b == -1) {
      if (new_vel) {
        const float4 v0 = new_vel[orig];
        new_vel[orig] = make_float4(v0.x + force.x, v0.y + force.y, v0.z + force.z, v0.w + 0.f);
      }
    } else {
      p_force[orig] = make_float4(force.x, force.y, force.z, 0.f);
      p_torque[orig] = make_float4(torque.x, torque.y, torque.z, 0.f);
      if (p_count) p_count[orig] = ncol;
    }
  }
}

// FindAugmentedRealityCollisionsUniformGridKernel / ...Cell (Kernels/RB_UniformGridKernels.cu:
// 879-996): per sorted particle, the 27 neighbour cells of the scene grid in z, y, x order;
// a scene point deepens the contact when 2r - d exceeds the deepest so far (starting from the
// caller's contact_distance), which records the distance and the point's cloud index at the
// particle's original index.  Colour green when any contact, else blue (color4 may be NULL).
__global__ void __launch_bounds__(128) static_find_kernel(
    ar_sim_params prm, ar_grid::Grid g, const float4* __restrict__ spos,
    const float4* __restrict__ scene_spos, const uint32_t* __restrict__ gidx,
    const uint32_t* __restrict__ scene_gidx, const uint32_t* __restrict__ cstart,
    const uint32_t* __restrict__ cend, int n, float* __restrict__ contact_distance,
    int32_t* __restrict__ contact_point, float4* __restrict__ color) {
  for (int index = blockIdx.x * blockDim.x + threadIdx.x; index < n;
       index += gridDim.x * blockDim.x) {
    const float3 pos = ar::xyz(__ldg(spos + index));
    const int3 gp = g.cell_of(pos);
    const uint32_t orig = __ldg(gidx + index);
    const float thr = 2 * prm.particle_radius;
    float deepest = contact_distance[orig];
    int best = contact_point[orig];
    int counter = 0;
    for (int z = -1; z <= 1; ++z)
      for (int y = -1; y <= 1; ++y)
        for (int x = -1; x <= 1; ++x) {
          const uint32_t h = g.hash(make_int3(gp.x + x, gp.y + y, gp.z + z));
          const uint32_t st = __ldg(cstart + h);
          if (st == ar::kEmpty) continue;
          const uint32_t en = __ldg(cend + h);
          for (uint32_t j = st; j < en; ++j) {
            const float3 d = ar::sub(pos, ar::xyz(__ldg(scene_spos + j)));
            const float dist = sqrtf(ar::dot(d, d));
            if (thr - dist > deepest) {
              deepest = thr - dist;
              best = (int)__ldg(scene_gidx + j);
              ++counter;
            }
          }
        }
    contact_distance[orig] = deepest;
    contact_point[orig] = best;
    if (color)
      color[orig] = counter ? make_float4(0.f, 1.f, 0.f, 0.f) : make_float4(0.f, 0.f, 1.f, 0.f);
  }
}

// GatherAugmentedRealityCollisions (Particles/updateFunctions.cpp:1511-1578) on the device: one
// contact per particle whose contact distance is positive, in particle order (an
// order-preserving compaction: a block-wide exclusive scan of the flags plus one atomic per
// block for the block's base, then a second kernel writes the contacts in block order).
// normal = the scene point's normal, point = rel + centre of the particle's body, body2 = -1,
// bias = ARrestitution * ((v + w x rel) . n); the accumulated impulses start at zero.
constexpr int kGatherThreads = 256;

__global__ void __launch_bounds__(kGatherThreads) static_gather_count_kernel(
    const float* __restrict__ contact_distance, int n, int32_t* __restrict__ block_counts) {
  __shared__ int s_count;
  if (threadIdx.x == 0) s_count = 0;
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool hit = i < n && contact_distance[i] > 0;
  const unsigned m = __ballot_sync(0xffffffffu, hit);
  if ((threadIdx.x & 31) == 0 && m) atomicAdd(&s_count, __popc(m));
  __syncthreads();
  if (threadIdx.x == 0) block_counts[blockIdx.x] = s_count;
}

// Exclusive scan of the per-block counts in one block (sequential over chunks of the block).
__global__ void __launch_bounds__(1024) static_gather_scan_kernel(int32_t* __restrict__ counts,
                                                                  int blocks,
                                                                  int32_t* __restrict__ total) {
  __shared__ int32_t s[1024];
  __shared__ int32_t carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < blocks; base += 1024) {
    const int i = base + threadIdx.x;
    const int32_t v = i < blocks ? counts[i] : 0;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
      const int32_t add = threadIdx.x >= o ? s[threadIdx.x - o] : 0;
      __syncthreads();
      s[threadIdx.x] += add;
      __syncthreads();
    }
    if (i < blocks) counts[i] = carry + s[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += s[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

__global__ void __launch_bounds__(kGatherThreads) static_gather_write_kernel(
    float restitution, int n, const int32_t* __restrict__ rb_idx, const float4* __restrict__ cms,
    const float4* __restrict__ vel, const float4* __restrict__ ang,
    const float4* __restrict__ rel4, const float4* __restrict__ scene_normals,
    const float* __restrict__ contact_distance, const int32_t* __restrict__ contact_point,
    const int32_t* __restrict__ block_base, int capacity, float4* __restrict__ normal,
    float4* __restrict__ point, int32_t* __restrict__ body1, int32_t* __restrict__ body2,
    float* __restrict__ bias, float* __restrict__ acc0, float* __restrict__ acc1,
    float* __restrict__ acc2, int* __restrict__ err) {
  __shared__ int32_t s_warp[kGatherThreads / 32];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool hit = i < n && contact_distance[i] > 0;
  const unsigned m = __ballot_sync(0xffffffffu, hit);
  if (lane == 0) s_warp[warp] = __popc(m);
  __syncthreads();
  int before = 0;
  for (int w = 0; w < warp; ++w) before += s_warp[w];
  if (!hit) return;
  const int c = block_base[blockIdx.x] + before + __popc(m & ((1u << lane) - 1));
  if (c >= capacity) {
    ar::raise_error(err, ar::kErrOverflow);
    return;
  }
  const int b = rb_idx[i];
  const float4 n4 = __ldg(scene_normals + contact_point[i]);
  const float4 r4 = __ldg(rel4 + i);
  const float4 cm = __ldg(cms + b);
  const float3 v = ar::xyz(__ldg(vel + b)), w = ar::xyz(__ldg(ang + b));
  const float3 r = ar::xyz(r4), nn = ar::xyz(n4);
  const float v_rel = ar::dot(ar::add(v, ar::cross(w, r)), nn);
  normal[c] = n4;
  point[c] = make_float4(r4.x + cm.x, r4.y + cm.y, r4.z + cm.z, r4.w + cm.w);
  body1[c] = b;
  body2[c] = -1;
  bias[c] = restitution * v_rel;
  acc0[c] = 0.f;
  acc1[c] = 0.f;
  acc2[c] = 0.f;
}

ar_status static_grid(const ar_sim_params* params, ar_grid::Grid* g) {
  *g = ar_grid::Grid::from_params(*params);
  for (uint32_t v : {g->gx, g->gy, g->gz})
    if (v == 0 || (v & (v - 1))) {
      arh::set_error("grid sizes must be powers of two");
      return AR_ERR_INVALID_ARG;
    }
  return AR_OK;
}

}  // namespace

extern "C" {

ar_status ar_collide_static_scene_impulse(
    ar_ctx* ctx, const ar_sim_params* params, const int32_t* rb_idx, const float* rel4,
    const float* inertia9, const float* mass, const float* scene_radii, const float* sorted_pos4,
    const float* sorted_vel4, const float* scene_sorted_pos4, const uint32_t* grid_idx,
    const uint32_t* scene_grid_idx, const uint32_t* scene_cell_start,
    const uint32_t* scene_cell_end, int n, float* p_force4, float* p_torque4,
    int32_t* p_count, float* new_vel4, float* color4, ar_stream_t stream) {
  if (!ctx || !params || n < 0 ||
      (n > 0 && (!rb_idx || !rel4 || !inertia9 || !mass || !scene_radii || !sorted_pos4 ||
                 !sorted_vel4 || !scene_sorted_pos4 || !grid_idx || !scene_grid_idx ||
                 !scene_cell_start || !scene_cell_end || !p_force4 || !p_torque4)))
    return AR_ERR_INVALID_ARG;
  ar_grid::Grid g;
  ar_status s = static_grid(params, &g);
  if (s != AR_OK || n == 0) return s;
  const unsigned grid = std::min(arh::grid_for(n, 128), (unsigned)ctx->num_sms * 16);
  static_impulse_kernel<<<grid, 128, 0, arh::stream(stream)>>>(
      *params, g, rb_idx, (const float4*)rel4, inertia9, mass, scene_radii,
      (const float4*)sorted_pos4, (const float4*)sorted_vel4, (const float4*)scene_sorted_pos4,
      grid_idx, scene_grid_idx, scene_cell_start, scene_cell_end, n, (float4*)p_force4,
      (float4*)p_torque4, p_count, (float4*)new_vel4, (float4*)color4);
  return arh::check_launch("ar_collide_static_scene_impulse");
}

ar_status ar_find_contacts_static_scene(ar_ctx* ctx, const ar_sim_params* params,
                                        const float* sorted_pos4,
                                        const float* scene_sorted_pos4,
                                        const uint32_t* grid_idx,
                                        const uint32_t* scene_grid_idx,
                                        const uint32_t* scene_cell_start,
                                        const uint32_t* scene_cell_end, int n,
                                        float* contact_distance, int32_t* contact_point,
                                        float* color4, ar_stream_t stream) {
  if (!ctx || !params || n < 0 ||
      (n > 0 && (!sorted_pos4 || !scene_sorted_pos4 || !grid_idx || !scene_grid_idx ||
                 !scene_cell_start || !scene_cell_end || !contact_distance || !contact_point)))
    return AR_ERR_INVALID_ARG;
  ar_grid::Grid g;
  ar_status s = static_grid(params, &g);
  if (s != AR_OK || n == 0) return s;
  const unsigned grid = std::min(arh::grid_for(n, 128), (unsigned)ctx->num_sms * 16);
  static_find_kernel<<<grid, 128, 0, arh::stream(stream)>>>(
      *params, g, (const float4*)sorted_pos4, (const float4*)scene_sorted_pos4, grid_idx,
      scene_grid_idx, scene_cell_start, scene_cell_end, n, contact_distance, contact_point,
      (float4*)color4);
  return arh::check_launch("ar_find_contacts_static_scene");
}

ar_status ar_gather_static_contacts(ar_ctx* ctx, const ar_sim_params* params, int n,
                                    const int32_t* rb_idx, const float* cms4, const float* vel4,
                                    const float* ang4, const float* rel4,
                                    const float* scene_normals4, const float* contact_distance,
                                    const int32_t* contact_point, int capacity, float* normal4,
                                    float* point4, int32_t* body1, int32_t* body2, float* bias,
                                    float* acc_impulse, float* acc_friction,
                                    float* acc_friction2, int32_t* d_count,
                                    ar_stream_t stream) {
  if (!ctx || !params || n < 0 || capacity < 0 || !d_count ||
      (n > 0 && (!rb_idx || !cms4 || !vel4 || !ang4 || !rel4 || !scene_normals4 ||
                 !contact_distance || !contact_point || !normal4 || !point4 || !body1 ||
                 !body2 || !bias || !acc_impulse || !acc_friction || !acc_friction2)))
    return AR_ERR_INVALID_ARG;
  cudaStream_t st = arh::stream(stream);
  if (n == 0) {
    cudaMemsetAsync(d_count, 0, sizeof(int32_t), st);
    return arh::check_launch("ar_gather_static_contacts");
  }
  const int blocks = (int)arh::grid_for(n, kGatherThreads);
  int32_t* base = (int32_t*)arh::scratch(ctx, (size_t)blocks * sizeof(int32_t) + 256);
  if (!base) return AR_ERR_OOM;
  static_gather_count_kernel<<<blocks, kGatherThreads, 0, st>>>(contact_distance, n, base);
  static_gather_scan_kernel<<<1, 1024, 0, st>>>(base, blocks, d_count);
  static_gather_write_kernel<<<blocks, kGatherThreads, 0, st>>>(
      params->ar_restitution, n, rb_idx, (const float4*)cms4, (const float4*)vel4,
      (const float4*)ang4, (const float4*)rel4, (const float4*)scene_normals4, contact_distance,
      contact_point, base, capacity, (float4*)normal4, (float4*)point4, body1, body2, bias,
      acc_impulse, acc_friction, acc_friction2, ctx->d_err);
  return arh::check_launch("ar_gather_static_contacts");
}

}  // extern "C"
