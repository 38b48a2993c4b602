// (a16/a17) per-body reduction, (a2) reference integrator, (a4) reference re-posing,
// (a18) reference wall collisions.
#include "ar_internal.cuh"
#include "ar_body.cuh"
#include "ar_glm.cuh"

namespace {

// ---- fixed-order segmented sum, one warp per body ---------------------------------------------
__global__ void __launch_bounds__(256) reduce_kernel(const float4* __restrict__ pf,
                                                     const float4* __restrict__ pt,
                                                     const int32_t* __restrict__ off, int nb,
                                                     float4* __restrict__ bf,
                                                     float4* __restrict__ bt) {
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < nb; b += warps) {
    float3 f, t;
    ar_body::warp_segment_sum(pf, pt, __ldg(off + b), __ldg(off + b + 1), &f, &t);
    if (ar::lane_id() == 0) {
      bf[b] = make_float4(f.x, f.y, f.z, 0.f);
      bt[b] = make_float4(t.x, t.y, t.z, 0.f);
    }
  }
}

// ReducePerParticleImpulses / CombineReducedImpulses (UniformGridDEM.cu:421-460) on top of the
// segmented sum: vel += F / m (float4 / float), ang += I^-1 tau (glm mat3 * vec3).
__global__ void __launch_bounds__(256) reduce_impulses_kernel(
    const float4* __restrict__ pf, const float4* __restrict__ pt, const int32_t* __restrict__ off,
    int nb, float4* __restrict__ vel, float4* __restrict__ ang, const float* __restrict__ mass,
    const float* __restrict__ inv_inertia) {
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < nb; b += warps) {
    float3 f, t;
    ar_body::warp_segment_sum(pf, pt, __ldg(off + b), __ldg(off + b + 1), &f, &t);
    if (ar::lane_id() == 0) {
      const float m = mass[b];
      float4 v = vel[b];
      vel[b] = make_float4(v.x + f.x / m, v.y + f.y / m, v.z + f.z / m, v.w + 0.f / m);
      float I[9];
      for (int k = 0; k < 9; ++k) I[k] = inv_inertia[9 * b + k];
      const float3 w = ar_glm::mv(I, t);
      float4 a = ang[b];
      ang[b] = make_float4(a.x + w.x, a.y + w.y, a.z + w.z, a.w + 0.f);
    }
  }
}

// ---- GPUintegratorKernel (Kernels/rigidBodyKernels.cu:262-348) ---------------------------------
__global__ void __launch_bounds__(128) integrate_reference_kernel(
    float3 gravity, float w_damping, float dt, int nb, float4* __restrict__ cms,
    float4* __restrict__ vel, float4* __restrict__ ang, float4* __restrict__ quat,
    const float* __restrict__ inv_inertia, float* __restrict__ cur_inertia,
    float* __restrict__ model, float4* __restrict__ cum_quat) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  float4 p = cms[b];
  float4 v = vel[b];
  const float4 w4 = ang[b];
  p = make_float4(p.x + v.x * dt, p.y + v.y * dt, p.z + v.z * dt, p.w + v.w * dt);
  const float3 nv = ar::mk3(w4.x, w4.y, w4.z);
  const float d = ar_glm::dot3(nv, nv);
  const float inv = 1.0f / sqrtf(d);  // glm::inversesqrt
  const float3 nrm = ar::mk3(nv.x * inv, nv.y * inv, nv.z * inv);
  const float theta = sqrtf(d) * dt;
  float4 q;
  if (theta > 0.00001f) {
    const float c = cosf(theta / 2.f), s = sinf(theta / 2.f);
    q = make_float4(s * nrm.x, s * nrm.y, s * nrm.z, c);
  } else {
    q = make_float4(0.f, 0.f, 0.f, 1.f);
  }
  q = ar_glm::qnormalize(q);
  float R[9], I[9], RI[9], Rt[9], C[9];
  ar_glm::mat3_cast(q, R);
  for (int k = 0; k < 9; ++k) I[k] = inv_inertia[9 * b + k];
  ar_glm::mm(R, I, RI);
  ar_glm::transpose(R, Rt);
  ar_glm::mm(RI, Rt, C);
  for (int k = 0; k < 9; ++k) cur_inertia[9 * b + k] = C[k];
  if (cum_quat) {
    float4 cq = ar_glm::qnormalize(ar_glm::qmul(q, cum_quat[b]));
    cum_quat[b] = cq;
    if (model) {
      float M[9];
      ar_glm::mat3_cast(cq, M);
      float* mo = model + 16 * b;
      for (int c = 0; c < 3; ++c) {
        for (int r = 0; r < 3; ++r) mo[c * 4 + r] = M[c * 3 + r];
        mo[c * 4 + 3] = 0.f;
      }
      mo[12] = p.x;
      mo[13] = p.y;
      mo[14] = p.z;
      mo[15] = 1.f;
    }
  }
  v = make_float4(v.x + gravity.x, v.y + gravity.y, v.z + gravity.z, v.w + 0.f);
  cms[b] = p;
  vel[b] = v;
  quat[b] = q;
  ang[b] = make_float4(nv.x * w_damping, nv.y * w_damping, nv.z * w_damping, 0.f * w_damping);
}

// ---- computeGlobalAttributes (rigidBodyKernels.cu:386-421) -------------------------------------
__global__ void __launch_bounds__(256) global_attributes_kernel(
    int n, const float4* __restrict__ cms, const float4* __restrict__ rb_vel,
    const float4* __restrict__ rb_ang, const float4* __restrict__ quat,
    const int32_t* __restrict__ rb_idx, float4* __restrict__ rel, float4* __restrict__ pos,
    float4* __restrict__ vel) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int b = __ldg(rb_idx + i);
  if (b == -1) return;
  float R[9];
  ar_glm::mat3_cast(__ldg(quat + b), R);
  const float4 r0 = rel[i];
  const float3 r = ar_glm::rotate_mat4(R, ar::mk3(r0.x, r0.y, r0.z));
  rel[i] = make_float4(r.x, r.y, r.z, 0.f);
  const float4 c = __ldg(cms + b);
  pos[i] = make_float4(r.x + c.x, r.y + c.y, r.z + c.z, 0.f + c.w);
  const float4 v = __ldg(rb_vel + b);
  const float3 w = ar::cross(ar::xyz(__ldg(rb_ang + b)), r);
  vel[i] = make_float4(v.x + w.x, v.y + w.y, v.z + w.z, v.w + 0.f);
}

__global__ void reset_quat_kernel(int nb, float4* __restrict__ quat) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b < nb) quat[b] = make_float4(0.f, 0.f, 0.f, 1.f);
}

// ---- integrateRigidBody (Kernels/rigidBodyKernels.cu:40-166): momentum form with box clamp --
struct MomentumArgs {
  float4 *cms, *vel, *force, *ang, *quat, *torque, *ang_mom, *lin_mom;
  const float* inv_inertia;
  float* cur_inertia;
  float* ang_acc;  // glm::vec3 per body
  const float *radii, *mass;
};

__global__ void __launch_bounds__(128) integrate_momentum_kernel(MomentumArgs a, float dt,
                                                                 float3 mn, float3 mx,
                                                                 float3 gravity, float bdamp,
                                                                 float gdamp, int nb) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  float4 L = a.lin_mom[b];
  const float4 F = a.force[b];
  L = make_float4(L.x + F.x * dt, L.y + F.y * dt, L.z + F.z * dt, L.w + F.w * dt);
  L = make_float4(L.x + gravity.x * dt, L.y + gravity.y * dt, L.z + gravity.z * dt, L.w + 0.f * dt);
  // the box is widened by double-precision literals, as written in the reference
  mx.x = (float)((double)mx.x + 0.1); mx.y = (float)((double)mx.y + 0.1); mx.z = (float)((double)mx.z + 0.1);
  mn.x = (float)((double)mn.x - 0.1); mn.y = (float)((double)mn.y - 0.1); mn.z = mn.z - 1;
  float4 p = a.cms[b];
  const float m = a.mass[b], r = a.radii[b];
  if (p.x > mx.x - r) { p.x = mx.x - r; L.x *= bdamp; }
  if (p.x < mn.x + r) { p.x = mn.x + r; L.x *= bdamp; }
  if (p.y > mx.y - r && L.y > 0) { p.y = mx.y - 2 * r; L.y *= bdamp; }
  if (p.y < mn.y + r) { p.y = mn.y + r; L.y *= bdamp; }
  if (p.z > mx.z - r) { p.z = mx.z - r; L.z *= bdamp; }
  if (p.z < mn.z + r) { p.z = mn.z + r; L.z *= bdamp; }
  L = make_float4(L.x * gdamp, L.y * gdamp, L.z * gdamp, L.w * gdamp);
  float4 v = make_float4(L.x * m, L.y * m, L.z * m, L.w * m);
  a.lin_mom[b] = L;
  p = make_float4(p.x + v.x * dt, p.y + v.y * dt, p.z + v.z * dt, p.w + v.w * dt);
  p.w = 0.f;
  v.w = 0.f;
  a.cms[b] = p;
  a.vel[b] = v;
  a.force[b] = make_float4(0.f, 0.f, 0.f, 0.f);
  float4 q = a.quat[b];
  float R[9], I[9], RI[9], Rt[9], C[9];
  ar_glm::mat3_cast(q, R);
  for (int k = 0; k < 9; ++k) I[k] = a.inv_inertia[9 * b + k];
  ar_glm::mm(R, I, RI);
  ar_glm::transpose(R, Rt);
  ar_glm::mm(RI, Rt, C);
  float4 am = a.ang_mom[b];
  const float4 tq = a.torque[b];
  am = make_float4(am.x + tq.x * dt, am.y + tq.y * dt, am.z + tq.z * dt, am.w + tq.w * dt);
  const float3 cm3 = ar::mk3(am.x, am.y, am.z);
  float3 nv = ar_glm::mv(C, cm3);
  const float3 acc = ar_glm::mv(C, ar_glm::cross3(cm3, nv));
  float4 qd = ar_glm::qmul(make_float4(nv.x, nv.y, nv.z, 0.f), q);  // glm::quat(0, w) * q
  qd = make_float4(qd.x / 2.f, qd.y / 2.f, qd.z / 2.f, qd.w / 2.f);
  q = make_float4(q.x + qd.x * dt, q.y + qd.y * dt, q.z + qd.z * dt, q.w + qd.w * dt);
  q = ar_glm::qnormalize(q);
  nv = ar::mk3(nv.x - acc.x * dt, nv.y - acc.y * dt, nv.z - acc.z * dt);
  if (a.ang_acc) {
    a.ang_acc[3 * b] = acc.x; a.ang_acc[3 * b + 1] = acc.y; a.ang_acc[3 * b + 2] = acc.z;
  }
  for (int k = 0; k < 9; ++k) a.cur_inertia[9 * b + k] = C[k];
  a.ang_mom[b] = am;
  a.quat[b] = q;
  a.ang[b] = make_float4(nv.x, nv.y, nv.z, 0.f);
  a.torque[b] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// ---- integrate_functor (Kernels/particleKernels.cu:50-128): free particles only -------------
__global__ void __launch_bounds__(256) integrate_particles_kernel(
    float4* __restrict__ pos, float4* __restrict__ vel, const int32_t* __restrict__ rb_idx,
    int n, float dt, float3 mn, float3 mx, float3 gravity, float gdamp, float bdamp, float r) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (rb_idx[i] >= 0) return;  // particles of rigid bodies are moved by their body
  const float4 p4 = pos[i], v4 = vel[i];
  float3 p = ar::mk3(p4.x, p4.y, p4.z), v = ar::mk3(v4.x, v4.y, v4.z);
  v = ar::add(v, ar::mk3(gravity.x * dt, gravity.y * dt, gravity.z * dt));
  v = ar::mk3(v.x * gdamp, v.y * gdamp, v.z * gdamp);
  p = ar::add(p, ar::mk3(v.x * dt, v.y * dt, v.z * dt));
  mx.x = (float)((double)mx.x + 0.01); mx.y = (float)((double)mx.y + 0.01); mx.z = (float)((double)mx.z + 0.01);
  mn.x = (float)((double)mn.x - 0.01); mn.y = (float)((double)mn.y - 0.01); mn.z = (float)((double)mn.z - 0.01);
  if (p.x > mx.x - r) { p.x = mx.x - r; v.x *= bdamp; }
  if (p.x < mn.x + r) { p.x = mn.x + r; v.x *= bdamp; }
  if (p.y > mx.y - r && v.y > 0) { p.y = mx.y - r; v.y *= bdamp; }
  if (p.z > mx.z - r) { p.z = mx.z - r; v.z *= bdamp; }
  if (p.z < mn.z + r) { p.z = mn.z + r; v.z *= bdamp; }
  if (p.y < mn.y + r) { p.y = mn.y + r; v.y *= bdamp; }
  pos[i] = make_float4(p.x, p.y, p.z, p4.w);
  vel[i] = make_float4(v.x, v.y, v.z, v4.w);
}

// ---- ReduceRigidBodyVariables (Kernels/rigidBodyKernels.cu:861-1043): per rigid object
// rb_force += sum(p_force), rb_torque += sum(p_torque) over [start, start + count); a non-finite
// sum raises the NaN error (the reference sets *toExit).
__global__ void __launch_bounds__(256) reduce_rbvars_kernel(
    const float4* __restrict__ pf, const float4* __restrict__ pt, const int32_t* __restrict__ start,
    const int32_t* __restrict__ count, int nb, float4* __restrict__ bf, float4* __restrict__ bt,
    int* __restrict__ err) {
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < nb; b += warps) {
    const int s = __ldg(start + b);
    float3 f, t;
    ar_body::warp_segment_sum(pf, pt, s, s + __ldg(count + b), &f, &t);
    if (ar::lane_id() == 0) {
      if (!isfinite(f.x + f.y + f.z) || !isfinite(t.x + t.y + t.z)) ar::raise_error(err, ar::kErrNaN);
      float4 a = bf[b], c = bt[b];
      bf[b] = make_float4(a.x + f.x, a.y + f.y, a.z + f.z, a.w);
      bt[b] = make_float4(c.x + t.x, c.y + t.y, c.z + t.z, c.w);
    }
  }
}

// ---- WallCollisionWrapper (WallCollisions.cu:46-90, 95-129, 201-276, 338-597) -------------------
struct Walls {
  float pos[6];  // wall position per plane, planes +x, +y, +z, -x, -y, -z
};

__device__ __forceinline__ float4 wall_normal(int w) {
  const float s = w < 3 ? 1.f : -1.f;
  const int a = w % 3;
  return make_float4(a == 0 ? s : 0.f, a == 1 ? s : 0.f, a == 2 ? s : 0.f, 0.f);
}
__device__ __forceinline__ float dot4(float4 a, float4 b) {
  return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w;
}

__global__ void __launch_bounds__(256) walls_reference_kernel(
    float radius, Walls walls, const float4* __restrict__ ppos, const float4* __restrict__ rbpos,
    float4* __restrict__ rbvel, float4* __restrict__ rbang, const float* __restrict__ inv_inertia,
    const float* __restrict__ mass, const int32_t* __restrict__ rb_idx,
    const int32_t* __restrict__ off, int nb) {
  const int warps = (gridDim.x * blockDim.x) >> 5;
  const int lane = ar::lane_id();
  for (int b = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; b < nb; b += warps) {
    const int s = __ldg(off + b), e = __ldg(off + b + 1);
    // DetectWallCollisionKernel x6: per particle the deepest admissible wall (distance starts
    // at 0: the wrapper memsets it, :372)
    float best_d = 0.f;
    int best_i = -1, best_w = 0;
    for (int i = s + lane; i < e; i += 32) {
      const int body = __ldg(rb_idx + i);
      if (body == -1) continue;
      const float4 v = rbvel[body];
      const float4 p = __ldg(ppos + i);
      float cd = 0.f;
      int cw = -1;
      for (int w = 0; w < 6; ++w) {
        const float4 nrm = wall_normal(w);
        const float sign = nrm.x * 1.f + nrm.y * 1.f + nrm.z * 1.f + nrm.w * 0.f;
        const float4 nn = make_float4(nrm.x * sign, nrm.y * sign, nrm.z * sign, nrm.w * sign);
        const float dist = sign * (dot4(p, nn) - walls.pos[w] + radius * sign);
        if (dist > cd && dot4(v, nrm) > 0.f) {
          cd = dist;
          cw = w;
        }
      }
      // per body: largest distance, ties -> larger particle index (the reference's three
      // stable sorts leave the last equal key at the segment end, WallCollisions.cu:533-537)
      // (a lane visits its particles in increasing index order, so >= keeps the later one)
      if (cw >= 0 && (best_i < 0 || cd >= best_d)) {
        best_d = cd;
        best_i = i;
        best_w = cw;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const float od = __shfl_xor_sync(0xffffffffu, best_d, o);
      const int oi = __shfl_xor_sync(0xffffffffu, best_i, o);
      const int ow = __shfl_xor_sync(0xffffffffu, best_w, o);
      if (oi >= 0 && (best_i < 0 || od > best_d || (od == best_d && oi > best_i))) {
        best_d = od;
        best_i = oi;
        best_w = ow;
      }
    }
    if (lane != 0 || best_i < 0 || !(best_d > 0.f)) continue;
    // HandleWallCollisionKernelUnmapped
    const float4 n = wall_normal(best_w);
    const float4 wall = make_float4(n.x * walls.pos[best_w], n.y * walls.pos[best_w],
                                    n.z * walls.pos[best_w], n.w * walls.pos[best_w]);
    const float4 p = __ldg(ppos + best_i);
    const float pd = dot4(p, n);
    const float4 paux = make_float4(n.x * pd, n.y * pd, n.z * pd, n.w * pd);
    const float4 ocm = rbpos[b];
    const float4 ov = rbvel[b];
    const float4 oa = rbang[b];
    float I[9];
    for (int k = 0; k < 9; ++k) I[k] = inv_inertia[9 * b + k];
    const float m = mass[b];
    const float4 disp = make_float4(p.x - ocm.x, p.y - ocm.y, p.z - ocm.z, p.w - ocm.w);
    const float4 rn = make_float4(radius * n.x, radius * n.y, radius * n.z, radius * n.w);
    const float4 ncm = make_float4(((ocm.x + wall.x) - rn.x) - paux.x, ((ocm.y + wall.y) - rn.y) - paux.y,
                                   ((ocm.z + wall.z) - rn.z) - paux.z, ((ocm.w + wall.w) - rn.w) - paux.w);
    float4 np = make_float4(ncm.x + disp.x, ncm.y + disp.y, ncm.z + disp.z, 1.f);
    // FindExactContactPointKernel(newP, newP + n r, r, 0)
    const float4 p2 = make_float4(np.x + n.x * radius, np.y + n.y * radius, np.z + n.z * radius,
                                  np.w + n.w * radius);
    const float t = radius / (radius + 0.f);
    const float4 dp = make_float4(p2.x - np.x, p2.y - np.y, p2.z - np.z, p2.w - np.w);
    const float4 cp = make_float4(np.x + dp.x * t, np.y + dp.y * t, np.z + dp.z * t, np.w + dp.w * t);
    const float il = 1.0f / sqrtf(dot4(dp, dp));
    const float4 cn = make_float4(dp.x * il * -1.f, dp.y * il * -1.f, dp.z * il * -1.f, dp.w * il * -1.f);
    const float4 r = make_float4(ncm.x - cp.x, ncm.y - cp.y, ncm.z - cp.z, ncm.w - cp.w);
    // ComputeImpulseMagnitudeKernel (:108-129)
    const float3 v3 = ar::mk3(ov.x, ov.y, ov.z), w3 = ar::mk3(oa.x, oa.y, oa.z);
    const float3 r3 = ar::mk3(r.x, r.y, r.z), n3 = ar::mk3(cn.x, cn.y, cn.z);
    const float3 va = ar::add(v3, ar_glm::cross3(w3, r3));
    const float numer = -(1.f + 1.f) * ar_glm::dot3(va, n3);
    const float a = 1.f / m;
    const float bb = ar_glm::dot3(ar_glm::cross3(ar_glm::mv(I, ar_glm::cross3(r3, n3)), r3), n3);
    const float j = numer / (a + bb);
    const float4 lin = make_float4(cn.x * j, cn.y * j, cn.z * j, cn.w * j);
    const float3 ai = ar_glm::mv(I, ar_glm::cross3(r3, ar::mk3(lin.x, lin.y, lin.z)));
    rbvel[b] = make_float4(ov.x + lin.x / m, ov.y + lin.y / m, ov.z + lin.z / m, ov.w + lin.w / m);
    rbang[b] = make_float4(oa.x + ai.x, oa.y + ai.y, oa.z + ai.z, oa.w + 0.f);
  }
}

unsigned warp_grid(const ar_ctx* ctx, int nb, int block) {
  long g = ((long)nb * 32 + block - 1) / block;
  long cap = (long)ctx->num_sms * 16;
  if (g > cap) g = cap;
  return (unsigned)(g < 1 ? 1 : g);
}

}  // namespace

extern "C" {

ar_status ar_reduce_bodies(ar_ctx* ctx, const float* p_force4, const float* p_torque4,
                           const int32_t* offsets, int num_bodies, float* body_force4,
                           float* body_torque4, ar_stream_t stream) {
  if (!ctx || num_bodies < 0 ||
      (num_bodies > 0 && (!p_force4 || !p_torque4 || !offsets || !body_force4 || !body_torque4)))
    return AR_ERR_INVALID_ARG;
  if (num_bodies == 0) return AR_OK;
  reduce_kernel<<<warp_grid(ctx, num_bodies, 256), 256, 0, arh::stream(stream)>>>(
      (const float4*)p_force4, (const float4*)p_torque4, offsets, num_bodies,
      (float4*)body_force4, (float4*)body_torque4);
  return arh::check_launch("ar_reduce_bodies");
}

ar_status ar_reduce_impulses(ar_ctx* ctx, const float* p_force4, const float* p_torque4,
                             const int32_t* offsets, int num_bodies, float* rb_vel4,
                             float* rb_ang4, const float* rb_mass, const float* rb_inv_inertia9,
                             ar_stream_t stream) {
  if (!ctx || num_bodies < 0 ||
      (num_bodies > 0 && (!p_force4 || !p_torque4 || !offsets || !rb_vel4 || !rb_ang4 ||
                          !rb_mass || !rb_inv_inertia9)))
    return AR_ERR_INVALID_ARG;
  if (num_bodies == 0) return AR_OK;
  reduce_impulses_kernel<<<warp_grid(ctx, num_bodies, 256), 256, 0, arh::stream(stream)>>>(
      (const float4*)p_force4, (const float4*)p_torque4, offsets, num_bodies, (float4*)rb_vel4,
      (float4*)rb_ang4, rb_mass, rb_inv_inertia9);
  return arh::check_launch("ar_reduce_impulses");
}

ar_status ar_integrate_reference(ar_ctx* ctx, const ar_sim_params* params, float dt,
                                 int num_bodies, float* cms4, float* vel4, float* ang4,
                                 float* quat4, const float* inv_inertia9,
                                 float* cur_inv_inertia9, float* model16, float* cum_quat4,
                                 const float* mass, ar_stream_t stream) {
  (void)mass;  // read but unused by the reference kernel (rigidBodyKernels.cu:283)
  if (!ctx || !params || num_bodies < 0 ||
      (num_bodies > 0 && (!cms4 || !vel4 || !ang4 || !quat4 || !inv_inertia9 ||
                          !cur_inv_inertia9)))
    return AR_ERR_INVALID_ARG;
  if (num_bodies == 0) return AR_OK;
  integrate_reference_kernel<<<arh::grid_for(num_bodies, 128), 128, 0, arh::stream(stream)>>>(
      make_float3(params->gravity[0], params->gravity[1], params->gravity[2]), params->w_damping,
      dt, num_bodies, (float4*)cms4, (float4*)vel4, (float4*)ang4, (float4*)quat4, inv_inertia9,
      cur_inv_inertia9, model16, (float4*)cum_quat4);
  return arh::check_launch("ar_integrate_reference");
}

ar_status ar_global_attributes(ar_ctx* ctx, int n, int num_bodies, const float* cms4,
                               const float* rb_vel4, const float* rb_ang4, float* quat4,
                               const int32_t* rb_idx, float* rel4, float* pos4, float* vel4,
                               ar_stream_t stream) {
  if (!ctx || n < 0 || num_bodies < 0 ||
      (n > 0 && (!cms4 || !rb_vel4 || !rb_ang4 || !quat4 || !rb_idx || !rel4 || !pos4 || !vel4)))
    return AR_ERR_INVALID_ARG;
  cudaStream_t st = arh::stream(stream);
  if (n > 0)
    global_attributes_kernel<<<arh::grid_for(n, 256), 256, 0, st>>>(
        n, (const float4*)cms4, (const float4*)rb_vel4, (const float4*)rb_ang4,
        (const float4*)quat4, rb_idx, (float4*)rel4, (float4*)pos4, (float4*)vel4);
  return arh::check_launch("ar_global_attributes");
}

ar_status ar_reset_quaternions(ar_ctx* ctx, float* quat4, int num_bodies, ar_stream_t stream) {
  if (!ctx || num_bodies < 0 || (num_bodies > 0 && !quat4)) return AR_ERR_INVALID_ARG;
  if (num_bodies > 0)
    reset_quat_kernel<<<arh::grid_for(num_bodies, 256), 256, 0, arh::stream(stream)>>>(
        num_bodies, (float4*)quat4);
  return arh::check_launch("ar_reset_quaternions");
}

ar_status ar_integrate_momentum(ar_ctx* ctx, const ar_sim_params* params, float dt,
                                int num_bodies, float* cms4, float* vel4, float* force4,
                                float* ang4, float* quat4, float* torque4, float* ang_mom4,
                                float* lin_mom4, const float* inv_inertia9,
                                float* cur_inv_inertia9, float* ang_acc3, const float* radii,
                                const float* mass, const float h_min_pos3[3],
                                const float h_max_pos3[3], ar_stream_t stream) {
  if (!ctx || !params || !h_min_pos3 || !h_max_pos3 || num_bodies < 0 ||
      (num_bodies > 0 && (!cms4 || !vel4 || !force4 || !ang4 || !quat4 || !torque4 ||
                          !ang_mom4 || !lin_mom4 || !inv_inertia9 || !cur_inv_inertia9 ||
                          !radii || !mass)))
    return AR_ERR_INVALID_ARG;
  if (num_bodies == 0) return AR_OK;
  MomentumArgs a{(float4*)cms4, (float4*)vel4, (float4*)force4, (float4*)ang4, (float4*)quat4,
                 (float4*)torque4, (float4*)ang_mom4, (float4*)lin_mom4, inv_inertia9,
                 cur_inv_inertia9, ang_acc3, radii, mass};
  integrate_momentum_kernel<<<arh::grid_for(num_bodies, 128), 128, 0, arh::stream(stream)>>>(
      a, dt, make_float3(h_min_pos3[0], h_min_pos3[1], h_min_pos3[2]),
      make_float3(h_max_pos3[0], h_max_pos3[1], h_max_pos3[2]),
      make_float3(params->gravity[0], params->gravity[1], params->gravity[2]),
      params->boundary_damping, params->global_damping, num_bodies);
  return arh::check_launch("ar_integrate_momentum");
}

ar_status ar_integrate_particles(ar_ctx* ctx, const ar_sim_params* params, float dt, float* pos4,
                                 float* vel4, const int32_t* rb_idx, int n,
                                 const float h_min_pos3[3], const float h_max_pos3[3],
                                 ar_stream_t stream) {
  if (!ctx || !params || !h_min_pos3 || !h_max_pos3 || n < 0 ||
      (n > 0 && (!pos4 || !vel4 || !rb_idx)))
    return AR_ERR_INVALID_ARG;
  if (n == 0) return AR_OK;
  integrate_particles_kernel<<<arh::grid_for(n, 256), 256, 0, arh::stream(stream)>>>(
      (float4*)pos4, (float4*)vel4, rb_idx, n, dt,
      make_float3(h_min_pos3[0], h_min_pos3[1], h_min_pos3[2]),
      make_float3(h_max_pos3[0], h_max_pos3[1], h_max_pos3[2]),
      make_float3(params->gravity[0], params->gravity[1], params->gravity[2]),
      params->global_damping, params->boundary_damping, params->particle_radius);
  return arh::check_launch("ar_integrate_particles");
}

ar_status ar_reduce_rigid_body_variables(ar_ctx* ctx, const float* p_force4,
                                         const float* p_torque4, const int32_t* starts,
                                         const int32_t* counts, int num_bodies,
                                         float* rb_force4, float* rb_torque4,
                                         ar_stream_t stream) {
  if (!ctx || num_bodies < 0 ||
      (num_bodies > 0 && (!p_force4 || !p_torque4 || !starts || !counts || !rb_force4 ||
                          !rb_torque4)))
    return AR_ERR_INVALID_ARG;
  if (num_bodies == 0) return AR_OK;
  reduce_rbvars_kernel<<<warp_grid(ctx, num_bodies, 256), 256, 0, arh::stream(stream)>>>(
      (const float4*)p_force4, (const float4*)p_torque4, starts, counts, num_bodies,
      (float4*)rb_force4, (float4*)rb_torque4, ctx->d_err);
  return arh::check_launch("ar_reduce_rigid_body_variables");
}

ar_status ar_walls_reference(ar_ctx* ctx, float radius, const float* particle_pos4,
                             const float* rb_pos4, const float h_min_pos3[3],
                             const float h_max_pos3[3], float* rb_vel4, float* rb_ang4,
                             const float* inv_inertia9, const float* rb_mass,
                             const int32_t* rb_idx, const int32_t* offsets, int num_bodies, int n,
                             ar_stream_t stream) {
  if (!ctx || !h_min_pos3 || !h_max_pos3 || num_bodies < 0 || n < 0 ||
      (num_bodies > 0 && (!particle_pos4 || !rb_pos4 || !rb_vel4 || !rb_ang4 || !inv_inertia9 ||
                          !rb_mass || !rb_idx || !offsets)))
    return AR_ERR_INVALID_ARG;
  if (num_bodies == 0) return AR_OK;
  // wall positions as the wrapper computes them (WallCollisions.cu:376-487)
  Walls w;
  for (int a = 0; a < 3; ++a) {
    w.pos[a] = h_max_pos3[a];
    w.pos[3 + a] = h_min_pos3[a];
  }
  walls_reference_kernel<<<warp_grid(ctx, num_bodies, 256), 256, 0, arh::stream(stream)>>>(
      radius, w, (const float4*)particle_pos4, (const float4*)rb_pos4, (float4*)rb_vel4,
      (float4*)rb_ang4, inv_inertia9, rb_mass, rb_idx, offsets, num_bodies);
  return arh::check_launch("ar_walls_reference");
}

}  // extern "C"
