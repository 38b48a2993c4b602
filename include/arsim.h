/*
 * arsim.h -- C ABI of libarsim.so, a B200 (sm_100a) implementation of AR_Sim's per-step
 * rigid-body pipeline (ATriantafyllopoulos/Diploma_Thesis).
 *
 * Conventions
 *  - Every entry point returns ar_status; none exits or aborts.  ar_last_error() gives the
 *    message of the last failure on the calling thread.
 *  - Array arguments are DEVICE pointers unless the name starts with `h_`.  Layouts are the
 *    reference's: "4" suffix = float4 per element (x, y, z, w) with w ignored on input,
 *    "9" = 3x3 matrix stored as glm::mat3 (column-major, 9 floats), quaternions are glm::quat
 *    memory order (x, y, z, w), AABB = 8 floats {min.x, min.y, min.z, max.x, max.y, max.z,
 *    pad, pad} (the reference's 16-byte aligned `struct AABB`, BVHSource/BVHcreation.h:33-37).
 *  - Work is enqueued on `stream` (a cudaStream_t; NULL = legacy default stream) and is
 *    asynchronous.  Nothing allocates or synchronises in steady state: temporaries come from
 *    the context's grow-only scratch arena, sized on first use.
 *  - Device-side failures (a bounded spin wait giving up, NaN state) set a word in the
 *    context that ar_ctx_status() reads back.
 *
 * Each declaration names the reference function it replaces (file:line within AR_Sim/).
 */
#ifndef ARSIM_H
#define ARSIM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AR_API __attribute__((visibility("default")))

typedef enum ar_status {
  AR_OK = 0,
  AR_ERR_INVALID_ARG = 1,
  AR_ERR_OOM = 2,
  AR_ERR_TIMEOUT = 3,     /* a device-side bounded wait gave up */
  AR_ERR_NAN = 4,         /* non-finite body state detected */
  AR_ERR_CUDA = 5,
  AR_ERR_UNSUPPORTED = 6,
  AR_ERR_OVERFLOW = 7     /* an output buffer (pair list) was too small */
} ar_status;

typedef void* ar_stream_t; /* cudaStream_t */

/* Simulation parameters.  Byte-for-byte the reference's `struct SimParams`
 * (Kernels/particleSystem.cuh:27-55), 128 bytes, so a SimParams* may be passed directly. */
typedef struct ar_sim_params {
  float collider_pos[3];
  float collider_radius;
  float gravity[3];
  float global_damping;
  float particle_radius;
  uint32_t grid_size[3];
  uint32_t num_cells;
  float world_origin[3];
  float cell_size[3];
  uint32_t num_bodies;
  uint32_t max_particles_per_cell;
  float spring;
  float damping;
  float shear;
  float attraction;
  float boundary_damping;
  float ar_restitution;
  float rb_restitution;
  float ar_friction;
  float rb_friction;
  float w_damping;
  float v_damping;
} ar_sim_params;

/* ---- context ------------------------------------------------------------------------- */
typedef struct ar_ctx ar_ctx;

/* Replaces the reference's implicit global CUDA state (cudaInit, Particles/
 * ParticleAuxiliaryFunctions.h:3) and its __constant__ SimParams (Kernels/particleKernels.cu:42).
 * Selects `device` and creates the per-device error word. */
AR_API ar_status ar_ctx_create(int device, ar_ctx** out);
AR_API ar_status ar_ctx_destroy(ar_ctx* ctx);
/* Synchronises `stream`, returns (and clears) any device-side error raised since the last
 * call: AR_ERR_TIMEOUT, AR_ERR_NAN, AR_ERR_OVERFLOW or AR_OK.  Replaces checkCudaErrors'
 * exit() (Libs/common/inc/helper_cuda.h:967-981). */
AR_API ar_status ar_ctx_status(ar_ctx* ctx, ar_stream_t stream);
/* Pre-size the scratch arena (so later calls inside a CUDA graph capture never grow it). */
AR_API ar_status ar_ctx_reserve(ar_ctx* ctx, size_t bytes);
AR_API const char* ar_last_error(void);
AR_API const char* ar_version(void);
/* Failure-detection test hook (no counterpart in the reference, whose allocation failures
 * exit through checkCudaErrors): after `after` more device or pinned-host allocations by this
 * library succeed, every later one fails on the host as if the memory were exhausted, so each
 * AR_ERR_OOM path can be exercised; `after` < 0 switches the injection off.  Process-wide. */
AR_API ar_status ar_test_fail_allocations(long after);

/* ---- (a6) scene bounding box -------------------------------------------------------------
 * findAABBCub (BVHSource/createMortonCodes.cu:65-107): min and max over all four lanes of
 * pos4[0..n), starting from +/-2139095040.0f (the reference's int `inf` macro, :10).
 * Writes one float4 each to d_min4 / d_max4 (device). */
AR_API ar_status ar_scene_aabb(ar_ctx* ctx, const float* pos4, int n, float* d_min4,
                               float* d_max4, ar_stream_t stream);

/* ---- (a7) Morton codes ---------------------------------------------------------------------
 * generateMortonCodes (BVHSource/BVHkernels.cu:646-716): normalise each position to the box,
 * 10 bits per axis, code = x*4 + y*2 + z interleave; idx[i] = i.  The box comes from device
 * memory (the createMortonCodes path, createMortonCodes.cu:109-251) ... */
AR_API ar_status ar_morton30(ar_ctx* ctx, const float* pos4, int n, const float* d_min4,
                             const float* d_max4, uint32_t* codes, int32_t* idx,
                             ar_stream_t stream);
/* ... or by value from the host (createMortonCodesPreallocated, createMortonCodes.cu:255-347). */
AR_API ar_status ar_morton30_box(ar_ctx* ctx, const float* pos4, int n, const float h_min4[4],
                                 const float h_max4[4], uint32_t* codes, int32_t* idx,
                                 ar_stream_t stream);
/* 63-bit variant (21 bits per axis), new: the reference only reserves CODE_LENGTH 21
 * (BVHSource/BVHkernels.cu:4-5).  Same normalisation, scale 2^21, clamp [0, 2^21-1]. */
AR_API ar_status ar_morton63(ar_ctx* ctx, const float* pos4, int n, const float* d_min4,
                             const float* d_max4, uint64_t* codes, int32_t* idx,
                             ar_stream_t stream);

/* ---- (a8) stable LSD radix sort ------------------------------------------------------------
 * Replaces cub::DeviceRadixSort::SortPairs (Kernels/particleKernelWrappers.cu:419-534,
 * BVHSource/createMortonCodes.cu:183-218).  Sorts (key, value) pairs by key bits
 * [begin_bit, end_bit) -- the reference always sorts all 32 bits; passing the number of
 * significant bits gives the same order with fewer passes.  Stable: equal keys keep input
 * order.  Inputs are left intact; results go to keys_out/vals_out (vals_in may be NULL to
 * mean the identity 0..n-1); the outputs must not overlap the inputs or each other
 * (AR_ERR_INVALID_ARG).  Onesweep: one histogram pass plus one pass per 8-bit digit
 * with decoupled look-back. */
AR_API ar_status ar_radix_sort_pairs_u32(ar_ctx* ctx, const uint32_t* keys_in,
                                         const uint32_t* vals_in, uint32_t* keys_out,
                                         uint32_t* vals_out, int n, int begin_bit, int end_bit,
                                         ar_stream_t stream);
AR_API ar_status ar_radix_sort_pairs_u64(ar_ctx* ctx, const uint64_t* keys_in,
                                         const uint32_t* vals_in, uint64_t* keys_out,
                                         uint32_t* vals_out, int n, int begin_bit, int end_bit,
                                         ar_stream_t stream);
/* ar_radix_sort_pairs_u32 with options (the same sort; cub::DeviceRadixSort::SortPairs has no
 * counterpart of these flags).
 *   AR_SORT_RANK_MATCH: rank each 8-bit digit with one warp match.any per item instead of a
 *     ballot per digit bit -- faster when the keys a warp holds share few digits (cell keys of
 *     particles stored body by body), slower when they share many (Morton codes).  The order
 *     is the same.
 *   AR_SORT_TEST_MUTE_FIRST_TILE: failure-detection test hook.  Tile 0 of every digit pass
 *     never publishes its look-back status, and the spin limit drops to 4,096 polls, so every
 *     later tile's look-back gives up: the device error word reports AR_ERR_TIMEOUT (read it
 *     with ar_ctx_status), the outputs are garbage, and nothing is written outside them. */
#define AR_SORT_RANK_MATCH 1u
#define AR_SORT_TEST_MUTE_FIRST_TILE 0x80000000u
AR_API ar_status ar_radix_sort_pairs_u32_ex(ar_ctx* ctx, const uint32_t* keys_in,
                                            const uint32_t* vals_in, uint32_t* keys_out,
                                            uint32_t* vals_out, int n, int begin_bit,
                                            int end_bit, uint32_t flags, ar_stream_t stream);

/* Allocation-free variant of ar_radix_sort_pairs_u32.  No counterpart in the reference.
 * For callers that cannot allocate device memory: a frame loop that must never stall on
 * cudaMalloc's implicit device synchronisation, code running while another component owns
 * the device memory pool, or a process whose device-memory budget is fixed at start-up.
 * The workspace is a static array inside libarsim.so (about 10 MiB, held by every GPU that
 * loads the library until the process exits), so n is limited to 1,048,576 pairs; larger n
 * returns AR_ERR_INVALID_ARG.  No context is needed and nothing is allocated: the caller
 * passes inputs and outputs, plus an optional device int (d_status, may be NULL) into which
 * a timed-out look-back ORs 1.  The first call on each device sets up (looks up the array's
 * device address with that device current); make that first call before any stream capture.
 * Every call on a device shares the array, so calls that overlap on the GPU race: serialise
 * them (one stream, or events).  The set-up is done once per device for the life of the
 * process and is not redone after cudaDeviceReset: do not call this entry point again in a
 * process that has reset the device.  Outputs must not overlap the inputs or each other. */
AR_API ar_status ar_radix_sort_pairs_u32_noalloc(const uint32_t* keys_in,
                                                 const uint32_t* vals_in, uint32_t* keys_out,
                                                 uint32_t* vals_out, int n, int begin_bit,
                                                 int end_bit, int32_t* d_status,
                                                 ar_stream_t stream);

/* ---- (a9) Karras LBVH hierarchy --------------------------------------------------------------
 * kernelConstructRadixTreeSoA (BVHSource/BVHSoAKernels.cu:7-99) with longestCommonPrefix
 * (BVHSource/BVHAuxiliary.cuh:31-43): leaves at [0, n), internal node i at n + i, root at n;
 * duplicate codes are tie-broken by the index prefix (clz(i ^ j) + 32).  Arrays have 2n-1
 * entries.  Writes is_leaf, left, right, parent, min_r, max_r of the internal nodes and the
 * parent of every node. */
AR_API ar_status ar_lbvh_build(ar_ctx* ctx, const uint32_t* sorted_codes, int n,
                               uint8_t* is_leaf, int32_t* left, int32_t* right,
                               int32_t* parent, int32_t* min_r, int32_t* max_r,
                               ar_stream_t stream);
/* 63-bit codes: same algorithm, prefix over 64 bits, ties broken by clz(i ^ j) + 64. */
AR_API ar_status ar_lbvh_build64(ar_ctx* ctx, const uint64_t* sorted_codes, int n,
                                 uint8_t* is_leaf, int32_t* left, int32_t* right,
                                 int32_t* parent, int32_t* min_r, int32_t* max_r,
                                 ar_stream_t stream);

/* ---- (a10) leaves ---------------------------------------------------------------------------
 * kernelConstructLeafNodesSoA + initializeRadii (BVHSoAKernels.cu:108-138,
 * Kernels/particleKernels.cu:694-708): leaf i gets is_leaf = 1, min_r = max_r = i,
 * cms4[i] = pos4[sorted_idx[i]], bounds[i] = cms +/- radius, radii[i] = radius. */
AR_API ar_status ar_lbvh_leaves(ar_ctx* ctx, int n, const int32_t* sorted_idx,
                                const float* pos4, float radius, uint8_t* is_leaf,
                                int32_t* min_r, int32_t* max_r, float* cms4, float* bounds8,
                                float* radii, ar_stream_t stream);

/* ---- (a11) bottom-up AABB refit --------------------------------------------------------------
 * kernelConstructInternalNodesSoA (BVHSoAKernels.cu:148-176): one thread per leaf climbs to
 * the root; the second thread to reach a node merges its children's boxes.  Unlike the
 * reference, the arrival counter has acquire-release semantics, so the merge always sees both
 * children's final boxes. */
AR_API ar_status ar_lbvh_refit(ar_ctx* ctx, int n, const int32_t* left, const int32_t* right,
                               const int32_t* parent, float* bounds8, ar_stream_t stream);


/* ---- (a12) BVH traversal ---------------------------------------------------------------------
 * collideBVHSoARigidBody (Kernels/RB_BVHKernels.cu:100-244) with collideStaticSpheresBVH
 * (:24-98): per sorted leaf, DEM force against every overlapping leaf of another body;
 * p_force4 / p_torque4 / p_positions4 are written at the particle's original index
 * (sorted_idx[leaf]); vel4 is the unsorted particle velocity.  Traversal is stackless
 * (parent links), so no per-thread stack limits the tree depth; `parent` may be NULL (the
 * reference's wrapper signature has none), in which case the links are derived from
 * left/right first.  Contacts are visited in the reference's order. */
AR_API ar_status ar_collide_bvh_dem(ar_ctx* ctx, const ar_sim_params* params,
                                    const int32_t* rb_idx, const float* rel4,
                                    const float* vel4, const uint8_t* is_leaf,
                                    const int32_t* left, const int32_t* right,
                                    const int32_t* parent, const float* cms4,
                                    const float* bounds8, const int32_t* sorted_idx,
                                    const float* radii, int n, float* p_force4,
                                    float* p_torque4, float* p_positions4, ar_stream_t stream);
/* FindRigidBodyCollisionsBVHKernel (Kernels/RB_BVHKernels.cu:760-876): per particle the
 * deepest contact with a later leaf (max_r >= leaf) of another body.  contact_distance is
 * read as the starting threshold and updated, like the reference. */
AR_API ar_status ar_find_contacts_bvh(ar_ctx* ctx, const int32_t* rb_idx,
                                      const uint8_t* is_leaf, const int32_t* left,
                                      const int32_t* right, const int32_t* parent,
                                      const int32_t* max_r, const float* cms4,
                                      const float* bounds8, const int32_t* sorted_idx,
                                      const float* radii, int n, float* contact_distance,
                                      int32_t* colliding_particle, int32_t* colliding_body,
                                      ar_stream_t stream);

/* Contact-pair sets (new; used to prove broad-phase equality).  Emits each unordered pair
 * {i, j} (original particle indices, i < j) with |p_i - p_j| < 2r and rb_idx[i] != rb_idx[j],
 * in unspecified order.  pairs2 holds capacity (i, j) int pairs; *d_count (device) receives
 * the number found; AR_ERR_OVERFLOW is raised through ar_ctx_status if it exceeds capacity. */
AR_API ar_status ar_pairs_bvh(ar_ctx* ctx, float radius, const int32_t* rb_idx,
                              const uint8_t* is_leaf, const int32_t* left,
                              const int32_t* right, const int32_t* parent, const float* cms4,
                              const float* bounds8, const int32_t* sorted_idx, int n,
                              int32_t* pairs2, int capacity, int32_t* d_count,
                              ar_stream_t stream);
AR_API ar_status ar_pairs_grid(ar_ctx* ctx, const ar_sim_params* params,
                               const int32_t* rb_idx, const float* sorted_pos4,
                               const uint32_t* grid_idx, const uint32_t* cell_start,
                               const uint32_t* cell_end, int n, int32_t* pairs2, int capacity,
                               int32_t* d_count, ar_stream_t stream);

/* ---- (a13) uniform-grid hash -----------------------------------------------------------------
 * calcHash / calcHashD (Kernels/particleKernelWrappers.cu:195-211, Kernels/particleKernels.cu:
 * 150-189): cell = floor((p - world_origin) / cell_size), wrapped with & (grid_size - 1)
 * (grid sizes must be powers of two), hash = z*Gy*Gx + y*Gx + x; idx[i] = i. */
AR_API ar_status ar_calc_hash(ar_ctx* ctx, const ar_sim_params* params, const float* pos4,
                              int n, uint32_t* hash, uint32_t* idx, ar_stream_t stream);

/* ---- (a14) reorder + cell ranges ---------------------------------------------------------------
 * reorderDataAndFindCellStart (Kernels/particleKernelWrappers.cu:213-254, kernel
 * Kernels/particleKernels.cu:193-258): clears cell_start[0..num_cells) to 0xffffffff, then
 * records the first/one-past-last sorted slot of every occupied cell and gathers
 * sorted_pos4/sorted_vel4 = pos4/vel4[sorted_idx].  cell_end is left stale for empty cells,
 * like the reference. */
AR_API ar_status ar_reorder_cells(ar_ctx* ctx, const uint32_t* sorted_hash,
                                  const uint32_t* sorted_idx, const float* pos4,
                                  const float* vel4, int n, uint32_t num_cells,
                                  uint32_t* cell_start, uint32_t* cell_end, float* sorted_pos4,
                                  float* sorted_vel4, ar_stream_t stream);

/* ---- depth-camera ingestion: the static scene's point cloud from a range image --------------
 * RGBDloader (Kernels/customRangeImageLoader.cu:14-113): per pixel (x, y) of a width x height
 * image of 16-bit depths (device memory; pixels whose index y * width + x exceeds
 * (width - 1) * (height - 1) are skipped, as in the reference): z = depth / 5000 (z < 0.01 ->
 * -1000), x' = z (x - 318.6) / 517.3, y' = z (y - 255.3) / 516.5, the point (x', y', z, 0) through
 * the transposed camera matrix (camera16: host, 16 floats, column-major glm::mat4) and the
 * reference's fixed gravity rotation, then (x, -y, -z) -> static_pos4 (w = 0), static_radii =
 * particle_radius, and vao5 (may be NULL) = x, y, z, x / width, y / height (the vertex records
 * the reference writes into its GL buffer).  Covers every pixel (the reference's launch only
 * whole 16 x 32 blocks). */
AR_API ar_status ar_range_image_cloud(ar_ctx* ctx, const uint16_t* depth, int width, int height,
                                      const float* camera16, float particle_radius,
                                      float* static_pos4, float* static_radii, float* vao5,
                                      ar_stream_t stream);

/* computeNormals (Kernels/customRangeImageLoader.cu:122-177): for every pixel not on the image
 * border, normal = normalize(cross(p(x, y+1) - p(x, y-1), p(x+1, y) - p(x-1, y))) with the
 * inverse length 1 / sqrtf (the reference's device build: rsqrtf); border pixels untouched. */
AR_API ar_status ar_range_image_normals(ar_ctx* ctx, const float* static_pos4, int width,
                                        int height, float* static_norm4, ar_stream_t stream);

/* ---- AR static scene (point cloud with normals) against the particles ---------------------
 * FindAndHandleAugmentedRealityCollisionsUniformGridKernel (RigidBodies/UniformGridDEM.cu:
 * 243-377): the scene's particles are hashed, sorted and given cell ranges with the same grid
 * (ar_calc_hash, ar_radix_sort_pairs_u32, ar_reorder_cells); then per sorted particle, the
 * scene particles in its 27 neighbour cells (z, y, x order) with d < 2r give
 *   I += -spring (2r - d) n + damping v_rel + shear v_t + attraction p_rel,
 * n = -(normal of the scene particle, unsorted, through scene_grid_idx), v_rel = -v; summed
 * per cell, then p_linear4[orig] += I, p_angular4[orig] += rel4[orig] x I, and color4[orig] =
 * (0, 1, 0, 0) when any contact (color4 may be NULL). */
AR_API ar_status ar_collide_static_scene_dem(ar_ctx* ctx, const ar_sim_params* params,
                                             const float* sorted_pos4, const float* sorted_vel4,
                                             const float* rel4, const float* scene_sorted_pos4,
                                             const float* scene_normals4,
                                             const uint32_t* grid_idx,
                                             const uint32_t* scene_grid_idx,
                                             const uint32_t* scene_cell_start,
                                             const uint32_t* scene_cell_end, int n,
                                             float* p_linear4, float* p_angular4,
                                             float* color4, ar_stream_t stream);

/* Impulse variant of the same collision (ARcollisionsUniformGridKernel with
 * collideARSpheresBaraffExact, Kernels/RB_UniformGridKernels.cu:420-667): per sorted particle,
 * for each scene point in its cell closer than r + scene_radii[point], an impulse
 * j = -(1 + ARrestitution) (v . n) / (((I^-1 (r_c x n)) x r_c) . n + 1/m) along n (the unit
 * vector from the point to the particle), r_c = contact point - body centre; p_force4[orig] and
 * p_torque4[orig] receive the sums and p_count[orig] the number of impulses (may be NULL).  As
 * in the reference, each of the 27 neighbour iterations examines the particle's own cell.
 * inertia9 / mass are the bodies' current inverse inertia and mass, indexed by rb_idx[orig].
 * A free particle (rb_idx -1) has its force added to new_vel4 instead (zero inverse inertia,
 * unit mass).  color4 (may be NULL): (0, 1, 0, 0) on any impulse. */
AR_API ar_status ar_collide_static_scene_impulse(
    ar_ctx* ctx, const ar_sim_params* params, const int32_t* rb_idx, const float* rel4,
    const float* inertia9, const float* mass, const float* scene_radii, const float* sorted_pos4,
    const float* sorted_vel4, const float* scene_sorted_pos4, const uint32_t* grid_idx,
    const uint32_t* scene_grid_idx, const uint32_t* scene_cell_start,
    const uint32_t* scene_cell_end, int n, float* p_force4, float* p_torque4, int32_t* p_count,
    float* new_vel4, float* color4, ar_stream_t stream);
/* Deepest contact of each particle with the static scene (FindAugmentedRealityCollisionsUniform-
 * GridKernel, Kernels/RB_UniformGridKernels.cu:879-996): 27 neighbour cells of the scene grid,
 * a point deepens the contact when 2r - d exceeds the current contact_distance[orig] (the
 * caller initialises it, 0 = none), which then records 2r - d and the point's cloud index in
 * contact_point[orig].  color4 (may be NULL): green on any contact, else blue. */
AR_API ar_status ar_find_contacts_static_scene(ar_ctx* ctx, const ar_sim_params* params,
                                               const float* sorted_pos4,
                                               const float* scene_sorted_pos4,
                                               const uint32_t* grid_idx,
                                               const uint32_t* scene_grid_idx,
                                               const uint32_t* scene_cell_start,
                                               const uint32_t* scene_cell_end, int n,
                                               float* contact_distance, int32_t* contact_point,
                                               float* color4, ar_stream_t stream);
/* GatherAugmentedRealityCollisions (Particles/updateFunctions.cpp:1511-1578) on the device: one
 * contact per particle with contact_distance > 0, in particle order: normal = scene_normals4 of
 * the contact point, point = rel + centre of the body, body1 = rb_idx, body2 = -1,
 * bias = ARrestitution ((v + w x rel) . n), accumulated impulses zero.  Writes the count to
 * d_count; more than `capacity` contacts raise AR_ERR_OVERFLOW (read with ar_ctx_status).  The
 * list feeds ar_sequential_impulse. */
AR_API ar_status ar_gather_static_contacts(ar_ctx* ctx, const ar_sim_params* params, int n,
                                           const int32_t* rb_idx, const float* cms4,
                                           const float* vel4, const float* ang4,
                                           const float* rel4, const float* scene_normals4,
                                           const float* contact_distance,
                                           const int32_t* contact_point, int capacity,
                                           float* normal4, float* point4, int32_t* body1,
                                           int32_t* body2, float* bias, float* acc_impulse,
                                           float* acc_friction, float* acc_friction2,
                                           int32_t* d_count, ar_stream_t stream);

/* Particles against the static scene through a BVH built over its point cloud (num_scene
 * leaves, built with ar_morton30 / ar_radix_sort_pairs_u32 / ar_lbvh_build / ar_lbvh_leaves /
 * ar_lbvh_refit; parent may be NULL), in the reference's visit order, leaves admitted by the
 * sphere-box test checkOverlap(float4, AABB, r) (BVHSource/BVHAuxiliary.cuh:159-175).
 * staticCollideBVHSoARigidBody (Kernels/RB_BVHKernels.cu:293-442): particle i (unsorted,
 * radius params.particle_radius) collects the DEM force of every overlapping leaf (the scene
 * point at rest, radius radii[leaf]) and rel x force into p_force4[i] / p_torque4[i]; the
 * reference adds them straight into the body's totals from many threads at once (racy), so
 * here the body sums are left to ar_reduce_bodies.  A free particle (rb_idx -1) gets v + force
 * in vel4 instead.  color4 (may be NULL): green when a leaf touches. */
AR_API ar_status ar_collide_bvh_static(ar_ctx* ctx, const ar_sim_params* params,
                                       const int32_t* rb_idx, const float* rel4,
                                       const float* pos4, float* vel4, const uint8_t* is_leaf,
                                       const int32_t* left, const int32_t* right,
                                       const int32_t* parent, const float* cms4,
                                       const float* bounds8, const float* radii, int num_scene,
                                       int n, float* p_force4, float* p_torque4, float* color4,
                                       ar_stream_t stream);
/* FindAugmentedRealityCollisionsBVHKernel (Kernels/RB_BVHKernels.cu:920-1023): deepest
 * contact of particle i with the scene through its tree: r + radii[point] - |cms[leaf] - p|
 * deeper than contact_distance[i] records it with the cloud point sorted_idx[leaf] in
 * contact_point[i].  The query radius is params.particle_radius (the reference reads the
 * scene's radius array at the query's index; the two agree when every radius is r).
 * color4 (may be NULL): green on a contact, white when none. */
AR_API ar_status ar_find_contacts_bvh_static(ar_ctx* ctx, const ar_sim_params* params,
                                             const float* pos4, const uint8_t* is_leaf,
                                             const int32_t* left, const int32_t* right,
                                             const int32_t* parent, const float* cms4,
                                             const float* bounds8, const int32_t* sorted_idx,
                                             const float* radii, int num_scene, int n,
                                             float* contact_distance, int32_t* contact_point,
                                             float* color4, ar_stream_t stream);

/* ---- (a15) DEM contact forces on the grid ------------------------------------------------------
 * FindAndHandleRigidBodyCollisionsUniformGridKernel (RigidBodies/UniformGridDEM.cu:57-241):
 * per sorted particle, the 27 neighbour cells in z, y, x order (-1..1), occupants in sorted
 * order, skipping itself and particles of its own body; for d < 2r:
 *   F += -spring (2r - d) n + damping v_rel + shear v_t + attraction p_rel
 * summed per cell then across cells; then p_force4[orig] += F and
 * p_torque4[orig] += rel4[orig] x F (accumulating, like the reference).  No atomics. */
AR_API ar_status ar_collide_grid_dem(ar_ctx* ctx, const ar_sim_params* params,
                                     const int32_t* rb_idx, const float* sorted_pos4,
                                     const float* sorted_vel4, const float* rel4,
                                     const uint32_t* grid_idx, const uint32_t* cell_start,
                                     const uint32_t* cell_end, int n, float* p_force4,
                                     float* p_torque4, ar_stream_t stream);

/* collideD / collideCell / collideSpheres (Kernels/particleKernels.cu:261-406), the particle
 * variant reached through collide() (Kernels/particleKernelWrappers.cu:256-305): same force
 * law, torque accumulated per cell (rel x cell force), results written (not accumulated) to
 * p_force4 / p_torque4 at the original index; particles with rb_idx -1 instead get
 * new_vel4[orig] = v + F (new_vel4 may be NULL when there are none). */
AR_API ar_status ar_collide_grid_particles(ar_ctx* ctx, const ar_sim_params* params,
                                           const int32_t* rb_idx, const float* sorted_pos4,
                                           const float* sorted_vel4, const float* rel4,
                                           const uint32_t* grid_idx,
                                           const uint32_t* cell_start,
                                           const uint32_t* cell_end, int n, float* p_force4,
                                           float* p_torque4, float* new_vel4,
                                           ar_stream_t stream);

/* ---- (a16/a17) per-body reduction --------------------------------------------------------------
 * Replaces ReducePerParticleImpulses + CombineReducedImpulses (RigidBodies/UniformGridDEM.cu:
 * 421-666) and ReduceRigidBodyVariables (Kernels/rigidBodyKernels.cu:861-1043): a fixed-order
 * segmented sum of p_force4 / p_torque4 over each body's particles [offsets[b], offsets[b+1])
 * (one warp per body: lane l sums elements l, l+32, ... in order, then a xor-shuffle tree
 * 16, 8, 4, 2, 1), written to body_force4 / body_torque4.  Deterministic and independent of
 * the other bodies.  The reference instead differences a global float prefix sum and reads
 * the segment start one element late (:440-441); this entry point sums each segment exactly
 * once. */
AR_API ar_status ar_reduce_bodies(ar_ctx* ctx, const float* p_force4, const float* p_torque4,
                                  const int32_t* offsets, int num_bodies, float* body_force4,
                                  float* body_torque4, ar_stream_t stream);
/* ReducePerParticleImpulses semantics on top of ar_reduce_bodies: rb_vel4 += F / mass,
 * rb_ang4 += inv_inertia9 * tau (CombineReducedImpulses, UniformGridDEM.cu:421-460). */
AR_API ar_status ar_reduce_impulses(ar_ctx* ctx, const float* p_force4, const float* p_torque4,
                                    const int32_t* offsets, int num_bodies, float* rb_vel4,
                                    float* rb_ang4, const float* rb_mass,
                                    const float* rb_inv_inertia9, ar_stream_t stream);

/* ReduceRigidBodyVariables (Kernels/rigidBodyKernels.cu:861-1043): for each rigid object b,
 * rb_force4[b] += sum and rb_torque4[b] += sum of p_force4 / p_torque4 over
 * [starts[b], starts[b] + counts[b]) (fixed order as above); a non-finite sum raises
 * AR_ERR_NAN through ar_ctx_status (the reference sets *toExit).  One launch for all bodies
 * instead of the reference's per-body host loop. */
AR_API ar_status ar_reduce_rigid_body_variables(ar_ctx* ctx, const float* p_force4,
                                                const float* p_torque4, const int32_t* starts,
                                                const int32_t* counts, int num_bodies,
                                                float* rb_force4, float* rb_torque4,
                                                ar_stream_t stream);

/* ---- (a2) body integration, reference semantics --------------------------------------------------
 * GPUintegratorKernel (Kernels/rigidBodyKernels.cu:262-348): x += v dt; q = axis-angle
 * rotation of omega*dt (identity below 1e-5 rad); current inverse inertia R I^-1 R^T;
 * cumulative quaternion and 4x4 model matrix; v += gravity (per step, no dt, as the
 * reference does); omega *= w_damping.  model16 / cum_quat4 may be NULL. */
AR_API ar_status ar_integrate_reference(ar_ctx* ctx, const ar_sim_params* params, float dt,
                                        int num_bodies, float* cms4, float* vel4, float* ang4,
                                        float* quat4, const float* inv_inertia9,
                                        float* cur_inv_inertia9, float* model16,
                                        float* cum_quat4, const float* mass,
                                        ar_stream_t stream);

/* ---- (a3) body integration, momentum form --------------------------------------------------------
 * integrateRigidBody / integrateSystemRigidBodies (Kernels/rigidBodyKernels.cu:40-210):
 * L += (F + g) dt with the box clamp (box widened by 0.1, 1.0 below in z) and boundary damping,
 * v = L * mass (the reference's rbMass holds 1/m on this path), x += v dt; angular momentum
 * += tau dt, w = R I^-1 R^T L, q += dt/2 (w,0) q normalised, w -= (R I^-1 R^T (L x w)) dt.
 * Force and torque are reset to zero.  ang_acc3 (glm::vec3 per body) may be NULL. */
AR_API ar_status ar_integrate_momentum(ar_ctx* ctx, const ar_sim_params* params, float dt,
                                       int num_bodies, float* cms4, float* vel4, float* force4,
                                       float* ang4, float* quat4, float* torque4,
                                       float* ang_mom4, float* lin_mom4,
                                       const float* inv_inertia9, float* cur_inv_inertia9,
                                       float* ang_acc3, const float* radii, const float* mass,
                                       const float h_min_pos3[3], const float h_max_pos3[3],
                                       ar_stream_t stream);

/* ---- (a4) particle re-posing, reference semantics -------------------------------------------------
 * computeGlobalAttributes (Kernels/rigidBodyKernels.cu:386-421): rel4 <- R(q) rel4 (in place),
 * pos4 = rel + cm, vel4 = v + omega x rel (particles with rb_idx -1 are skipped). */
AR_API ar_status ar_global_attributes(ar_ctx* ctx, int n, int num_bodies, const float* cms4,
                                      const float* rb_vel4, const float* rb_ang4, float* quat4,
                                      const int32_t* rb_idx, float* rel4, float* pos4,
                                      float* vel4, ar_stream_t stream);
/* resetQuaternionKernel (Kernels/rigidBodyKernels.cu:449-456): q <- identity. */
AR_API ar_status ar_reset_quaternions(ar_ctx* ctx, float* quat4, int num_bodies,
                                      ar_stream_t stream);

/* ---- (a5) free particles ----------------------------------------------------------------------------
 * integrate_functor / integrateSystem (Kernels/particleKernels.cu:50-148): for particles with
 * rb_idx == -1: v += g dt, v *= global_damping, x += v dt, clamped to the box widened by 0.01
 * with boundary_damping.  Particles of rigid bodies are untouched. */
AR_API ar_status ar_integrate_particles(ar_ctx* ctx, const ar_sim_params* params, float dt,
                                        float* pos4, float* vel4, const int32_t* rb_idx, int n,
                                        const float h_min_pos3[3], const float h_max_pos3[3],
                                        ar_stream_t stream);
/* initializeRadii (Kernels/particleKernels.cu:694-708) and similar fills: dst[0..n) = value. */
AR_API ar_status ar_fill_f32(ar_ctx* ctx, float* dst, long n, float value, ar_stream_t stream);

/* ---- (a18) wall collisions, reference semantics ---------------------------------------------------
 * WallCollisionWrapper (WallCollisions.cu:338-597): per particle the deepest of the six box
 * walls it penetrates while its body moves toward that wall (walls tested +x, +y, +z, -x, -y,
 * -z; a later wall must be strictly deeper); per body the deepest such contact (ties -> the
 * larger particle index); then a Baraff e = 1 impulse on the body's linear and angular
 * velocity (HandleWallCollisionKernelUnmapped, :201-276).  One gather per body, no sorts.
 * offsets[b]..offsets[b+1] are the body's particles. */
AR_API ar_status ar_walls_reference(ar_ctx* ctx, float radius, const float* particle_pos4,
                                    const float* rb_pos4, const float h_min_pos3[3],
                                    const float h_max_pos3[3], float* rb_vel4, float* rb_ang4,
                                    const float* inv_inertia9, const float* rb_mass,
                                    const int32_t* rb_idx, const int32_t* offsets,
                                    int num_bodies, int n, ar_stream_t stream);

/* ---- sequential-impulse path (updateUniformGridSIS, RigidBodies/UniformGridUpdate.cpp:734-815) ----
 * REFERENCE semantics, all on the device (the reference gathers and solves on the host).
 *
 * FindRigidBodyCollisionsUniformGridKernel (Kernels/RB_UniformGridKernels.cu:731-842): per
 * sorted particle over the 27 neighbour cells, the deepest penetration 2r - |p - q| by a
 * particle of another body that exceeds contact_distance[original index] (the running maximum:
 * zero it before the call, as the reference does), with that particle's original index and
 * body.  Inputs are ar_calc_hash / sort / ar_reorder_cells outputs. */
AR_API ar_status ar_find_contacts_grid(ar_ctx* ctx, const ar_sim_params* params,
                                       const int32_t* rb_idx, const float* sorted_pos4,
                                       const uint32_t* grid_idx, const uint32_t* cell_start,
                                       const uint32_t* cell_end, int n, float* contact_distance,
                                       int32_t* colliding_body, int32_t* colliding_particle,
                                       ar_stream_t stream);
/* GatherRigidBodyCollisions (Particles/updateFunctions.cpp:1431-1500): every particle with
 * contact_distance > 0, in particle order (particles stored body by body, rb_idx their
 * bodies), becomes contact c: point and normal of findExactContactPoint on CM + rel of the
 * two particles (float4 arithmetic, Particles/CPU_Engine.cpp:461-473), body1 = its body,
 * body2 = the colliding body, bias = rb_restitution * relative normal velocity, accumulated
 * impulse and frictions 0.  *d_count (device) receives the number of contacts; those beyond
 * capacity are dropped and raise AR_ERR_OVERFLOW through ar_ctx_status. */
AR_API ar_status ar_gather_contacts(ar_ctx* ctx, const ar_sim_params* params, int n,
                                    const int32_t* rb_idx, const float* cms4, const float* vel4,
                                    const float* ang4, const float* rel4,
                                    const float* contact_distance, const int32_t* colliding_body,
                                    const int32_t* colliding_particle, int capacity,
                                    float* normal4, float* point4, int32_t* body1,
                                    int32_t* body2, float* bias, float* acc_impulse,
                                    float* acc_friction, float* acc_friction2, int32_t* d_count,
                                    ar_stream_t stream);
/* SequentialImpulseSolver (Particles/updateFunctions.cpp:1580-1874): `iterations` (the
 * reference uses 18) Gauss-Seidel sweeps over the *d_count contacts in order; accumulated
 * impulse clamped to [0, 100], friction to +-friction * mc * |g.y| (ar_friction for one-body
 * contacts, body2 == -1, whose impulse includes friction; rb_friction for body pairs, whose
 * applied impulse is the normal part only, as in the reference); body velocities and angular
 * velocities updated in place.  Bit-identical to the sequential loop: contacts that share no
 * body are solved together, one dependency level at a time, in one thread block, and later
 * sweeps start before earlier ones end wherever no body is shared (each body still sees the
 * loop's order of updates).  iterations x (capacity + 1) must stay below 2^31
 * (AR_ERR_INVALID_ARG otherwise). */
AR_API ar_status ar_sequential_impulse(ar_ctx* ctx, const ar_sim_params* params,
                                       const int32_t* d_count, int capacity,
                                       const float* normal4, const float* point4,
                                       const int32_t* body1, const int32_t* body2,
                                       const float* bias, float* acc_impulse,
                                       float* acc_friction, float* acc_friction2,
                                       int num_bodies, const float* cms4, float* vel4,
                                       float* ang4, const float* cur_inv_inertia9,
                                       const float* mass, int iterations, ar_stream_t stream);

/* ==== fused step: scenes and batches ================================================================
 * A scene is one independent rigid-body world resident on the device.  ar_step advances it
 * with the fused pipeline (re-pose + hash, the order by (key, particle index) -- re-sorted
 * from the previous step's order, or radix-sorted in the first step after a change of the
 * member list -- scatter + cell ranges, DEM gather + walls, fixed-order body reduction +
 * integration), PHYSICAL semantics:
 *   v += (g + F/m) dt,  omega += I_w^-1 tau dt,  x += v dt,
 *   q += dt/2 (omega, 0) q, normalised;  I_w^-1 = R I_b^-1 R^T,
 * with box walls as DEM springs (the wall is a static sphere surface at the plane).
 * Body-frame particle offsets stay constant (no incremental re-rotation drift).
 * Replaces ParticleSystem::updateUniformGridDEM (RigidBodies/UniformGridUpdate.cpp:939-999)
 * and updateRigidBodies (RigidBodies/BVHUpdate.cpp:5-438). */

enum { AR_BROADPHASE_GRID = 0, AR_BROADPHASE_BVH = 1 };

typedef struct ar_scene_desc {
  int num_bodies;
  int num_particles;
  float radius;          /* particle radius r; contact distance 2r */
  float box_min[3];      /* walls */
  float box_max[3];
  float gravity[3];
  float dt;
  float spring;          /* k */
  float damping;         /* dashpot coefficient on relative velocity */
  float shear;           /* coefficient on tangential relative velocity */
  float attraction;
  int broadphase;        /* AR_BROADPHASE_GRID or AR_BROADPHASE_BVH */
  float cell_size;       /* grid cell edge; 0 -> 2r */
  int grid_log2[3];      /* log2 grid cells per axis (wrapped); 0 -> derived from the box */
  int block_size;        /* threads per CTA for the collision kernel: 0 -> 128 (grid) or 64
                            (BVH), else a multiple of 32 in [32, 256] */
} ar_scene_desc;

typedef struct ar_scene ar_scene;

/* Host-side initial state, all arrays host memory:
 *  body_pos4[B], body_quat4[B] (x,y,z,w), body_vel4[B], body_angvel4[B], body_mass[B],
 *  body_inv_inertia9[B] (body frame, glm::mat3 layout), body_offsets[B+1] (particles of body
 *  b are [off[b], off[b+1]), particle_rel4[N] (body-frame offsets from the body centre). */
typedef struct ar_scene_init {
  const float* body_pos4;
  const float* body_quat4;
  const float* body_vel4;
  const float* body_angvel4;
  const float* body_mass;
  const float* body_inv_inertia9;
  const int32_t* body_offsets;
  const float* particle_rel4;
} ar_scene_init;

AR_API ar_status ar_scene_create(ar_ctx* ctx, const ar_scene_desc* desc,
                                 const ar_scene_init* init, ar_stream_t stream,
                                 ar_scene** out);
AR_API ar_status ar_scene_destroy(ar_scene* scene);
/* A new scene with `proto`'s description and current state, copied on the device in stream
 * order (one device-to-device copy of the scene's block, no host synchronisation): the server
 * keeps request templates resident and admits a request by cloning its template.  `proto`
 * must not change until the copy has run on `stream`.  No counterpart in the reference (its
 * bodies are built on the host by ParticleSystem::addRigidBody). */
AR_API ar_status ar_scene_clone_async(const ar_scene* proto, ar_stream_t stream,
                                      ar_scene** out);
/* Release a scene's device memory in stream order (cudaFreeAsync on `stream`), without a
 * host or device-wide synchronisation.  Every use of the scene must be ordered before this
 * point of `stream` (e.g. the scene was removed from its batches before the batch's next step
 * on that stream).  Scene memory comes from the device's stream-ordered pool, so a server can
 * admit and retire scenes while steps run. */
AR_API ar_status ar_scene_destroy_async(ar_scene* scene, ar_stream_t stream);
/* Attach a static point cloud to a grid scene (the augmented-reality scene from
 * ar_range_image_cloud / ar_range_image_normals): cloud_pos4 and cloud_norm4 are device arrays
 * of num_points float4 (w ignored), copied into the library, sorted by cell of the scene's grid
 * and given their own cell table (8 bytes per cell of the scene's grid).  From the next step
 * on, every particle also takes the impulses of the cloud points within 2r, in the reference's
 * law (FindAndHandleAugmentedRealityCollisionsUniformGridKernel, RigidBodies/UniformGridDEM.cu:
 * 243-377: along the point's negated normal, the scene at rest), summed over the 27
 * neighbour cells in z, y, x order and added to the particle's force after its particle
 * contacts and walls -- the simulateAR branch of updateUniformGridDEM
 * (RigidBodies/UniformGridUpdate.cpp:967-969), which re-sorts the cloud every step; here it
 * is sorted once.  num_points = 0 detaches the cloud.  Synchronises the device (steps in
 * flight may read the old cloud); every batch holding the scene rebuilds its table before
 * its next step.  A clone (ar_scene_clone_async) starts without a cloud.  BVH scenes:
 * AR_ERR_INVALID_ARG. */
AR_API ar_status ar_scene_set_static_cloud(ar_ctx* ctx, ar_scene* scene, const float* cloud_pos4,
                                           const float* cloud_norm4, int num_points,
                                           ar_stream_t stream);
/* Device bytes a scene with this description keeps resident (state + its share of the
 * step workspace); used for HBM-budget admission. */
AR_API size_t ar_scene_footprint(const ar_scene_desc* desc);
/* Cells of the grid a scene with this description gets (0 for the BVH broad phase).  A
 * batch holds fewer than AR_MAX_BATCH_CELLS cells and AR_MAX_BATCH_PARTICLES particles in
 * total (cell keys and particle indices are 32-bit); ar_batch_step rejects larger batches. */
#define AR_MAX_BATCH_CELLS 4294967295ull
#define AR_MAX_BATCH_PARTICLES 1073741823
AR_API uint64_t ar_scene_cells(const ar_scene_desc* desc);
/* Copy body state to host arrays (any may be NULL); synchronises the stream. */
AR_API ar_status ar_scene_download(ar_scene* scene, float* h_body_pos4, float* h_body_quat4,
                                   float* h_body_vel4, float* h_body_angvel4,
                                   ar_stream_t stream);
/* The same without the synchronisation: the copies are queued on the stream (truly
 * asynchronous into pinned host memory); the arrays are valid once the stream has reached
 * this point. */
AR_API ar_status ar_scene_download_async(ar_scene* scene, float* h_body_pos4,
                                         float* h_body_quat4, float* h_body_vel4,
                                         float* h_body_angvel4, ar_stream_t stream);
/* Overwrite body state from host arrays (any may be NULL); asynchronous (use pinned memory
 * for overlap).  Replaces the reference's per-step host round trip of body state
 * (Particles/updateFunctions.cpp:2903-2930). */
AR_API ar_status ar_scene_upload(ar_scene* scene, const float* h_body_pos4,
                                 const float* h_body_quat4, const float* h_body_vel4,
                                 const float* h_body_angvel4, ar_stream_t stream);
/* Packed body state: h_state16 holds pos[nb], quat[nb], vel[nb], angvel[nb] back to back
 * (16 floats per body in all), moved with one contiguous copy each way instead of four.
 * ar_scene_upload_state is asynchronous (pinned memory for overlap);
 * ar_scene_download_state returns once the state is on the host, and
 * ar_scene_download_state_async once the copy is queued on `stream`.  Same role as
 * ar_scene_upload / ar_scene_download (Particles/updateFunctions.cpp:2903-2930). */
AR_API ar_status ar_scene_upload_state(ar_scene* scene, const float* h_state16,
                                       ar_stream_t stream);
AR_API ar_status ar_scene_download_state(ar_scene* scene, float* h_state16, ar_stream_t stream);
AR_API ar_status ar_scene_download_state_async(ar_scene* scene, float* h_state16,
                                               ar_stream_t stream);
/* A host round trip in one call: the packed body state is uploaded from h_state_in16, the
 * scene advances n_steps (CUDA graph), and its packed state is copied to h_state_out16 (both
 * pinned host memory; they may be the same array); returns once the state is on the host.
 * The reference's per-frame pattern -- state to the device, step, state back for the renderer
 * (Particles/updateFunctions.cpp:2903-2930) -- with one entry instead of three. */
AR_API ar_status ar_scene_step_io(ar_ctx* ctx, ar_scene* scene, const float* h_state_in16,
                                  int n_steps, float* h_state_out16, ar_stream_t stream);
/* Device pointers of the scene's resident arrays (for tests / zero-copy consumers). */
typedef struct ar_scene_view {
  int num_bodies, num_particles;
  float* body_pos4; float* body_quat4; float* body_vel4; float* body_angvel4;
  float* body_mass; float* body_inv_inertia9; int32_t* body_offsets;
  float* particle_rel4;           /* w holds the body index (int bits) */
  float* body_force4; float* body_torque4;   /* last step's per-body totals */
} ar_scene_view;
AR_API ar_status ar_scene_get_view(ar_scene* scene, ar_scene_view* out);

/* Grid the scene was given: origin, cell edge and cells per axis (powers of two). */
AR_API ar_status ar_scene_grid_info(ar_scene* scene, float origin[3], float cell[3],
                                    uint32_t dims[3]);

/* Device pointers into the workspace of the scene's last ar_step (for parity tests and
 * consumers that want the sorted state): the sorted keys and the particle index of each
 * sorted slot, sorted positions (w = body index, int bits) and velocities, the per-particle
 * DEM + wall force at the original index, and for the grid broad phase the cell table: two
 * uint32 per cell, {first sorted slot, meta}, meta = occupant count (bits 0-4, 31 meaning 31
 * or more) | step epoch (bits 5-12: the step number mod 255, plus 1; any other value marks an
 * empty cell) | body tag (bits 13-31: scene-local body + 1 when every occupant belongs to that
 * body, else 0).  Grid keys are uint32 cell keys
 * (key_bytes 4); BVH keys are the scene index above a 30-bit Morton code, uint32 when they
 * fit in 32 bits (at most 4 scenes; key_bytes 4) and uint64 otherwise (key_bytes 8), and the
 * BVH view adds the
 * tree (leaf i at i, internal node i at N + i, root N) and tree_nodes16: 16 floats per
 * internal node holding both children's boxes, ids and body tags -- left lo.xyz, hi.x |
 * hi.y, hi.z, left id, left tag | right lo.xyz, hi.x | hi.y, hi.z, right id, right tag (ids
 * and tags as int bits; a tag is the global body id when every leaf below that child belongs
 * to one body, else -1).  Tree pointers are NULL for the grid, cells2 NULL for the BVH. */
typedef struct ar_step_view {
  int num_particles;
  uint64_t num_cells;
  int key_bits;
  uint32_t* sorted_keys; /* uint64_t* when key_bytes == 8 */
  uint32_t* sorted_idx;
  float* sorted_pos4;
  float* sorted_vel4;
  float* particle_force4;
  uint32_t* cells2;
  int key_bytes;
  int broadphase;
  int32_t* tree_left;
  int32_t* tree_right;
  int32_t* tree_parent;
  float* tree_nodes16;
} ar_step_view;
AR_API ar_status ar_scene_step_view(ar_scene* scene, ar_step_view* out);

/* Advance one scene by n_steps (one launch sequence per step; captured into a CUDA graph on
 * first use when use_graph != 0). */
AR_API ar_status ar_step(ar_ctx* ctx, ar_scene* scene, int n_steps, int use_graph,
                         ar_stream_t stream);

/* Run n_steps of the scene without a graph, with CUDA events between the stages, and return
 * the average device milliseconds per stage in h_stage_ms[6].  Grid: clear (sort histogram
 * head), re-pose + cell keys + histogram, sort, scatter + cell table, DEM gather + walls, body
 * sums + integration (+ cell reset).  BVH: clear (refit counters), Morton keys, sort, tree
 * (build, leaves, scene roots, refit), DEM traversal + walls, body sums + integration.
 * (Replaces the reference's clock() accumulators, e.g.
 * RigidBodies/UniformGridUpdate.cpp:338-446.) */
AR_API ar_status ar_step_profile(ar_ctx* ctx, ar_scene* scene, int n_steps, float* h_stage_ms,
                                 ar_stream_t stream);

/* Per-particle DEM + wall force of the last step (original particle order): copies N float4
 * to a device buffer.  p_torque4 is reserved and may be NULL (torques are summed per body
 * from the forces, see ar_scene_view.body_torque4). */
AR_API ar_status ar_scene_particle_forces(ar_scene* scene, float* p_force4, float* p_torque4,
                                          ar_stream_t stream);

/* A batch advances many scenes with one launch per stage: keys of all scenes are sorted
 * together in a global cell space (scene cell base + local cell), every per-particle kernel
 * is a grid-stride loop over the concatenation, and the step is a CUDA graph.  Each scene's
 * result is bit-identical to stepping it alone. */
typedef struct ar_batch ar_batch;
AR_API ar_status ar_batch_create(ar_ctx* ctx, ar_batch** out);
AR_API ar_status ar_batch_destroy(ar_batch* batch);
/* Replace the batch's member list (scenes stay resident and owned by the caller).  All
 * scenes of a batch use one broad phase.  Changing the list costs no host synchronisation
 * unless the batch's workspace has to grow. */
AR_API ar_status ar_batch_set_scenes(ar_batch* batch, ar_scene* const* scenes, int n_scenes);
/* The same with a step budget per scene: scene i is integrated by at most steps_left[i] of the
 * batch's following steps (< 0: no limit) and is frozen afterwards -- it still takes part in
 * the broad phase, but its state no longer changes, so it may be read (or removed at the next
 * member change) while later steps run.  A frozen scene's state equals that of the scene
 * stepped alone steps_left[i] times.  Used by a server that steps fixed-size ticks. */
AR_API ar_status ar_batch_set_scenes_limited(ar_batch* batch, ar_scene* const* scenes,
                                             int n_scenes, const int64_t* steps_left);
AR_API ar_status ar_batch_step(ar_ctx* ctx, ar_batch* batch, int n_steps, int use_graph,
                               ar_stream_t stream);
/* ar_step_profile for a batch. */
AR_API ar_status ar_batch_profile(ar_ctx* ctx, ar_batch* batch, int n_steps,
                                  float* h_stage_ms, ar_stream_t stream);
/* Render hand-off (replaces the reference's modelMatrixGPU output of GPUintegratorKernel,
 * Kernels/rigidBodyKernels.cu:322-331, and its GL buffer): one glm::mat4 per body,
 * column-major (16 floats: mat3_cast of the orientation, translation = body centre), written
 * to a 16-byte aligned device buffer -- for a batch in member order, one launch. */
AR_API ar_status ar_batch_model_matrices(ar_batch* batch, float* d_model16, ar_stream_t stream);
AR_API ar_status ar_scene_model_matrices(ar_scene* scene, float* d_model16, ar_stream_t stream);

/* ---- continuous-batching server (no counterpart in the reference) ---------------------------
 * A request loop in C++ over the batch API.  A request names a template scene (uploaded once
 * with ar_server_add_template and kept resident) and a number of steps K, and arrives at a
 * given time (seconds from the start of ar_server_run, on the host's steady clock).  The loop
 * runs fixed ticks of tick_steps batch steps on its own stream:
 *   1. admission in arrival order while the requests' footprints (ar_scene_footprint) fit the
 *      HBM budget and the batch stays within AR_MAX_BATCH_* and max_batch_particles; an
 *      admitted request's scene is a clone of its template (ar_scene_clone_async) on an
 *      admission stream that the compute stream waits for -- no host synchronisation;
 *   2. one tick: ar_batch_set_scenes_limited (each scene's remaining K as its step budget, so a
 *      scene is frozen after exactly K steps) when the members changed, then ar_batch_step;
 *   3. a finished scene's state is copied to the host behind the tick (into the request's
 *      pinned buffer h_results[i] when given, in the layout of ar_scene_download_state: 16
 *      floats per body -- else into a scratch buffer) and the request completes
 *      when the host sees that copy done; the scene leaves the batch at the next member change
 *      and is freed in stream order (ar_scene_destroy_async).
 * The host runs at most max_inflight ticks ahead of the device.  Admission stops at
 * time_limit_s (< 0: no limit); requests not admitted by then are not completed. */
typedef struct ar_server ar_server;
typedef struct ar_server_stats {
  int completed, offered, peak_resident, ticks;
  double wall_s;
  long long scene_steps, particle_steps;
  size_t peak_bytes;
  double host_admit_s, host_set_s, host_step_s, host_retire_s, host_wait_s;
} ar_server_stats;
AR_API ar_status ar_server_create(ar_ctx* ctx, double hbm_budget_bytes, int tick_steps,
                                  long long max_batch_particles, int max_inflight,
                                  ar_server** out);
/* Uploads a template scene (ar_scene_create on the server's admission stream); *id receives
 * its index for ar_server_run. */
AR_API ar_status ar_server_add_template(ar_server* server, const ar_scene_desc* desc,
                                        const ar_scene_init* init, int* id);
/* Serves n requests (template_id[i], steps[i], arrival_s[i]; arrival order need not be
 * sorted).  latency_s[i] receives completion - arrival in seconds, or -1 for a request not
 * completed; h_results may be NULL, and so may any h_results[i]. */
AR_API ar_status ar_server_run(ar_server* server, int n, const int* template_id,
                               const int* steps, const double* arrival_s, double time_limit_s,
                               float* const* h_results, double* latency_s,
                               ar_server_stats* stats);
AR_API ar_status ar_server_destroy(ar_server* server);

/* Autotuner timing loop (no counterpart in the reference): the scene `init` is created under
 * each of the n_cand descriptions (candidate broad phase, cell size, wrapped grid and collision
 * block size), stepped `warmup` times (CUDA graph), then `steps` graph-replayed steps are timed
 * with CUDA events on a stream of its own; ms_per_step[i] receives candidate i's time.  The
 * caller picks the fastest; every candidate gives the same contacts. */
AR_API ar_status ar_tune_candidates(ar_ctx* ctx, const ar_scene_desc* descs, int n_cand,
                                    const ar_scene_init* init, int warmup, int steps,
                                    float* ms_per_step);

/* Number of kernel launches one step of this batch issues (for launch accounting). */
AR_API int ar_batch_launches_per_step(ar_batch* batch);
AR_API int ar_scene_launches_per_step(ar_scene* scene);

#ifdef __cplusplus
}
#endif
#endif /* ARSIM_H */
