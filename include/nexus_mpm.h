/*
 * nexus_mpm.h — C ABI of the B200 (sm_100a) MLS-MPM step.
 *
 * A drop-in for nexus_mpm's `MpmPipeline::step` and the `MpmState` /
 * `GpuParticles` calls around it (reference crate nexus_mpm3d 0.5.0).
 * Every entry point below names the reference interface it replaces
 * (path:line within the reference project).  Plain pointers and sizes
 * only; the library owns all device memory.
 *
 * Conventions
 *   - Return value: 0 (NXM_OK) or a negative NXM_E_* code.
 *   - Matrices are column-major, 9 floats (glam Mat3 layout).
 *   - A state is used by one host thread at a time; calls on one state are
 *     ordered on that state's CUDA stream.  nxm_step enqueues and returns;
 *     readbacks synchronize the state's stream.
 *   - Particle indices are stable: particle i stays at index i until it is
 *     removed (the sort reorders an index list, never the particle arrays).
 */
#ifndef NEXUS_MPM_H
#define NEXUS_MPM_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define NXM_API __attribute__((visibility("default")))
#else
#define NXM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- error codes ------------------------------------------------------- */
#define NXM_OK 0
#define NXM_E_INVALID (-1)      /* bad argument (null pointer, out-of-range index, ...) */
#define NXM_E_CUDA (-2)         /* a CUDA runtime call failed */
#define NXM_E_CAPACITY (-3)     /* more active grid blocks than the grid capacity */
#define NXM_E_HASH_FULL (-4)    /* the block hash map is full */
#define NXM_E_NO_DEVICE (-5)    /* no CUDA device / the library cannot run here */
#define NXM_E_UNSUPPORTED (-6)  /* a feature this build does not implement */
#define NXM_E_OOM (-7)          /* device allocation failed */

/* Device status bits reported by nxm_state_status (sticky until cleared). */
#define NXM_STATUS_HASH_FULL 1u
#define NXM_STATUS_BLOCK_CAPACITY 2u
#define NXM_STATUS_MISSING_BLOCK 4u
#define NXM_STATUS_SORT_CAPACITY 8u
#define NXM_STATUS_COPY_TIMEOUT 16u  /* a kernel's wait for its bulk copies ran out (reported as NXM_E_CUDA) */

/* ---- plain data -------------------------------------------------------- */

/* SimulationParams (src_mpm_shaders/solver/params.rs:9-17). */
typedef struct nxm_simulation_params {
    float gravity[3];
    float dt;
} nxm_simulation_params;

/* MpmCapacities (src_mpm/pipeline.rs:27-43): grid_size = grid blocks to
 * reserve (rounded up to a power of two, as GpuGrid::with_capacity does). */
typedef struct nxm_capacities {
    uint32_t grid_size;
    uint32_t particles_capacity;
} nxm_capacities;

/* GpuParticleModel (src_mpm_shaders/models/default.rs:41-44): tag + 24 words,
 * 100 bytes, bit-identical to the reference's host packing
 * (src_mpm/solver/particle_model.rs:282-325). */
typedef struct nxm_particle_model {
    uint32_t tag;
    uint32_t data[24];
} nxm_particle_model;

/* Particle + ParticleDynamics (src_mpm/solver/particle.rs:26-122). */
typedef struct nxm_particle {
    float position[3];
    float velocity[3];
    float def_grad[9];
    float affine[9];
    float force_dt[3];
    float vel_grad_det;
    float init_volume;
    float init_radius;
    float mass;
    float damping;
    float phase;
    float boundary_friction;
    uint32_t group_id;
    uint32_t enabled;
    uint32_t fixed;
    nxm_particle_model model;
} nxm_particle;

/* Structure-of-arrays view of n particles, for bulk upload (the same fields
 * as nxm_particle; any pointer except position and model may be NULL to
 * take the Particle::new default: zero velocity/affine/force/vel_grad_det,
 * identity F, damping 0, phase 1, boundary_friction 1, group 0, enabled 1,
 * fixed 0; init_volume/mass are then required; a missing init_radius is
 * taken from init_volume = (2 r)^3).  boundary_friction scales the colliders'
 * friction under CPIC; init_radius, phase and group_id only feed the render
 * data (nxm_prep_readback). */
typedef struct nxm_particles_soa {
    const float* position;        /* n*3 */
    const float* velocity;        /* n*3 */
    const float* def_grad;        /* n*9 */
    const float* affine;          /* n*9 */
    const float* vel_grad_det;    /* n   */
    const float* init_volume;     /* n   */
    const float* init_radius;     /* n   */
    const float* mass;            /* n   */
    const float* damping;         /* n   */
    const float* phase;           /* n   */
    const float* boundary_friction; /* n */
    const uint32_t* group_id;     /* n   */
    const uint32_t* enabled;      /* n   */
    const uint32_t* fixed;        /* n   */
    const nxm_particle_model* model; /* n */
} nxm_particles_soa;

/* BoundaryCondition (src_mpm_shaders/solver/boundary_condition.rs:105-115). */
#define NXM_BC_STICK 0u
#define NXM_BC_SLIP 1u
#define NXM_BC_SEPARATE 2u
#define NXM_BC_NON_REFLECTING 3u

/* One coupled collider (128 bytes): Shape (src_rbd_shaders/shapes/shape.rs:29-73;
 * shape_a[3] holds the bit pattern of the shape type: 0 ball, 1 cuboid,
 * 2 capsule, 6 trimesh), Pose3 (rotation quaternion x,y,z,w + translation),
 * Velocity (src_rbd_shaders/dynamics/body.rs:216-225), local centre of mass,
 * BoundaryCondition, and for a trimesh the range of its triangles in the
 * triangle buffer passed to nxm_state_set_colliders. */
typedef struct nxm_collider {
    float shape_a[4];
    float shape_b[4];
    float shape_c[4];
    float rotation[4];
    float translation[3];
    float linvel[3];
    float angvel[3];
    float local_com[3];
    uint32_t bc_type;
    float bc_friction;
    uint32_t tri_first;
    uint32_t tri_count;
} nxm_collider;

/* Per-phase device times of the last timed step (GpuTimestamps,
 * src_mpm/pipeline.rs:389-524), milliseconds. */
typedef struct nxm_timestamps {
    float sort_ms;
    float p2g_ms;
    float grid_update_ms;
    float g2p_ms;   /* G2P and particle update (one fused kernel) */
    float total_ms;
} nxm_timestamps;

typedef struct nxm_pipeline nxm_pipeline;
typedef struct nxm_state nxm_state;

/* ---- pipeline ------------------------------------------------------------ */

/* MpmPipeline::new (src_mpm/pipeline.rs:366-382).  Checks for an sm_100
 * device; there is no CPU fallback. */
NXM_API int nxm_pipeline_create(nxm_pipeline** out);
NXM_API void nxm_pipeline_destroy(nxm_pipeline* pipeline);

/* MpmPipeline::step (src_mpm/pipeline.rs:385-526): sort, P2G, grid update
 * (with collider projection unless CPIC is on), G2P + particle update,
 * body integration.  Enqueued on the state's stream; returns immediately.
 * `timestamps` may be NULL; when given, the call waits and fills it. */
NXM_API int nxm_step(nxm_pipeline* pipeline, nxm_state* state, nxm_timestamps* timestamps);

/* ---- state -------------------------------------------------------------- */

/* MpmState::empty (src_mpm/pipeline.rs:107-165): no particles, cell width
 * 1, dt = 1/60, zero gravity. */
NXM_API int nxm_state_create(const nxm_capacities* capacities, nxm_state** out);
NXM_API void nxm_state_destroy(nxm_state* state);

/* MpmState::set_simulation_params (src_mpm/pipeline.rs:169-178). */
NXM_API int nxm_state_set_simulation_params(nxm_state* state, const nxm_simulation_params* params);

/* MpmState::write_substep_params (src_mpm/pipeline.rs:183-196): dt = base_dt / max(substeps, 1). */
NXM_API int nxm_state_write_substep_params(nxm_state* state, uint32_t num_substeps);

/* MpmState::set_cell_width (src_mpm/pipeline.rs:200-209). */
NXM_API int nxm_state_set_cell_width(nxm_state* state, float cell_width, uint32_t grid_capacity);

/* MpmState::set_coupling (src_mpm/pipeline.rs:220-247) for one-way coupled
 * colliders given directly (at most 16).  `tri_vertices` holds 3 vertices
 * (9 floats) per triangle, in the local frame of the owning trimesh; a
 * trimesh collider uses triangles [tri_first, tri_first + tri_count), for
 * which the library builds a BVH and the feature pseudo-normals (the
 * reference uploads both from its host mesh, rbd shapes/trimesh.rs).  Unlike
 * the reference, this does not switch CPIC on; see nxm_state_set_use_cpic. */
NXM_API int nxm_state_set_colliders(nxm_state* state, const nxm_collider* colliders, uint32_t num_colliders,
                            const float* tri_vertices, uint32_t num_triangles);

/* Overwrites the velocity of collider i (kinematic driving, e.g. velocity =
 * d(pose)/dt each step; the step integrates the pose from it).  Ordered on
 * the state's stream before the next step, without a host synchronisation
 * (the values travel as kernel arguments). */
NXM_API int nxm_state_set_collider_velocity(nxm_state* state, uint32_t index, const float linvel[3], const float angvel[3]);

/* Kinematic driving of colliders [first, first + count) at once: 6 floats
 * each (linear then angular velocity).  Ordered on the state's stream before
 * the next step, without a host synchronisation (the source array may be
 * reused as soon as the call returns).  No reference counterpart: the
 * reference writes body velocities one buffer at a time. */
NXM_API int nxm_state_set_collider_velocities(nxm_state* state, uint32_t first, uint32_t count, const float* vel6);

/* Reads collider i's pose: quaternion x,y,z,w then translation (7 floats). */
NXM_API int nxm_state_read_collider_pose(nxm_state* state, uint32_t index, float out[7]);

/* MpmState::use_cpic (src_mpm/pipeline.rs:69): CPIC coupling with the
 * colliders (node and particle distance fields, compatible / incompatible
 * P2G and G2P, penetration reprojection and penalty; two-way impulses off as
 * in the reference build).  Analytic colliders (ball, cuboid, capsule) enter
 * the node field directly (solver/grid_update_cdf.rs); trimesh colliders
 * through rigid particles sampled on their surface at the cell width
 * (sampling/sample_trimesh.rs, resampled when the colliders or the cell width
 * change), moved with the collider pose each step, sorted into the blocks
 * and projected on the nodes (solver/rigid_particle_update.rs,
 * grid/sort.rs:165-249 and 493-667, solver/p2g_cdf.rs); in batched-scene
 * mode each scene's samples take its block-key region and its colliders'
 * scene-local affinity bits (every scene's samples are rebuilt when a scene
 * is added or removed).  CPIC keeps particles in id order; deterministic
 * mode runs the gather-form transfers, the fast mode a scatter P2G with the
 * compatible / incompatible split. */
NXM_API int nxm_state_set_use_cpic(nxm_state* state, int enabled);
/* Number of CPIC rigid particles (GpuRigidParticles::len,
 * src_mpm/solver/particle.rs:351-354); 0 without CPIC or trimesh colliders. */
NXM_API int nxm_state_num_rigid_particles(const nxm_state* state, uint32_t* count);
/* The CPIC rigid particles in sampling order: local position xyz, owning
 * collider (u32 bits), triangle index inside that collider's range (u32
 * bits), 5 floats each (the reference's sample_points + sample_ids,
 * sampling/sample_trimesh.rs:33-56). */
NXM_API int nxm_read_rigid_particles(nxm_state* state, float* out);

/* Render data, headless (src_mpm/solver/prep_readback.rs, shader
 * src_mpm_shaders/solver/prep_readback.rs).  RenderConfig modes: */
#define NXM_RENDER_DEFAULT 0u       /* the group color */
#define NXM_RENDER_VOLUME 1u        /* (1 - singular values of F) / 0.005 + 0.2 */
#define NXM_RENDER_VELOCITY 2u      /* |v| dt 100 + 0.2 */
#define NXM_RENDER_PHASE 3u         /* (0, 0.4 phase, 0.4 (1 - phase)) */
#define NXM_RENDER_CDF_NORMALS 4u   /* (CPIC normal + 1) / 2 */
#define NXM_RENDER_CDF_DISTANCES 5u /* CPIC signed distance / 1.5 dx: green outside, red inside */
#define NXM_RENDER_CDF_SIGNS 6u     /* black: no affinity, green: no sign bit, red: a sign bit */

/* ReadbackData (prep_readback.rs:81-93, 3D): color rgba (alpha of the group
 * color; disabled particles (1, 0, 0, 1)), deformation diag(2 init_radius) *
 * clamp(F, -4, 4) as a column-major 4x4 (Mat4::from_mat3), position. */
typedef struct nxm_readback_data {
    float color[4];
    float deformation[16];
    float position[3];
    float pad;
} nxm_readback_data;

/* WgPrepReadback::launch (prep_readback.rs:152-200) for the particles: one
 * record per particle, in particle-id order, read back into `out`
 * (n records); synchronizes.  `palette` holds `num_groups` rgba colors
 * indexed by group_id modulo num_groups (NULL or 0: the reference's default
 * six-color palette). */
NXM_API int nxm_prep_readback(nxm_state* state, uint32_t mode, const float* palette, uint32_t num_groups,
                              nxm_readback_data* out);

/* WgPrepReadback::launch_render (gpu_mpm_prep_render): the same data written
 * straight into caller-owned DEVICE buffers, per particle in id order:
 * positions (3 floats), deformations (9, the column-major 3x3), colors (4,
 * 16-byte aligned); asynchronous on the state's stream (headless: plain CUDA
 * buffers where the reference writes a renderer's instance buffers). */
NXM_API int nxm_prep_render(nxm_state* state, uint32_t mode, const float* palette, uint32_t num_groups,
                            float* positions, float* deformations, float* colors);

/* gpu_prep_readback_rigid (prep_readback.rs:420-469): one record per CPIC
 * rigid particle (sampling order): base color (`colors`, 4 floats per rigid
 * particle, or NULL for the palette cycled over the particles as
 * GpuReadbackData::new does), deformation diag(0.4 cell width), world
 * position as of the start of the last step (the local sample before any
 * step); synchronizes. */
NXM_API int nxm_prep_readback_rigid(nxm_state* state, const float* colors, const float* palette,
                                    uint32_t num_groups, nxm_readback_data* out);
/* Particle Cdf (solver/particle.rs:35-50) of every particle: normal xyz,
 * signed distance, rigid velocity xyz, affinity bits (u32 bits), 8 floats
 * each; synchronizes. */
NXM_API int nxm_read_cdf(nxm_state* state, float* out);

/* Deterministic mode: canonical sort order (ascending id inside every sort
 * bucket) and the reference's atomic-free, gather-form P2G with its
 * summation order.  Off by default (the fast path scatters with atomics). */
NXM_API int nxm_state_set_deterministic(nxm_state* state, int enabled);

/* ---- particles -------------------------------------------------------- */

/* GpuParticles::append (src_mpm/solver/particle.rs:533-565). */
NXM_API int nxm_particles_append(nxm_state* state, const nxm_particle* particles, uint32_t count);
/* Same, from structure-of-arrays host buffers. */
NXM_API int nxm_particles_append_soa(nxm_state* state, const nxm_particles_soa* particles, uint32_t count);

/* GpuParticles::swap_remove (src_mpm/solver/particle.rs:579-631).  Writes up
 * to `count` (from, to) relocation pairs to `remaps` (may be NULL) and their
 * number to `num_remaps`. */
NXM_API int nxm_particles_swap_remove(nxm_state* state, const uint32_t* slots, uint32_t count, uint32_t* remaps,
                              uint32_t* num_remaps);

/* GpuParticles::shift_remove (src_mpm/solver/particle.rs:505-531) for [start, end). */
NXM_API int nxm_particles_shift_remove(nxm_state* state, uint32_t start, uint32_t end);

/* GpuParticles::len (src_mpm/solver/particle.rs:374-377). */
NXM_API uint32_t nxm_particles_len(const nxm_state* state);

/* GpuParticles::read_positions (src_mpm/solver/particle.rs:634-647) and the
 * other per-particle fields (n*3, n*3, n*9, n*9, n, n, n, n*25 words). */
NXM_API int nxm_read_positions(nxm_state* state, float* out);
NXM_API int nxm_read_velocities(nxm_state* state, float* out);
NXM_API int nxm_read_affine(nxm_state* state, float* out);
NXM_API int nxm_read_def_grad(nxm_state* state, float* out);
NXM_API int nxm_read_vel_grad_det(nxm_state* state, float* out);
NXM_API int nxm_read_mass(nxm_state* state, float* out);
NXM_API int nxm_read_enabled(nxm_state* state, uint32_t* out);
NXM_API int nxm_read_models(nxm_state* state, nxm_particle_model* out);

/* ---- grid inspection (parity tests, debugging) -------------------------- */

/* Number of active blocks of the last sort. */
NXM_API int nxm_grid_num_blocks(nxm_state* state, uint32_t* out);
/* Per block, in this build's header order, 23 int32: virtual id xyz,
 * first_particle, num_particles, num_particles_with_extras,
 * sort_bucket_cursors[10] (as left by the sort: bucket ends), nbh_block_ids[7]
 * (ActiveBlockHeader, src_mpm_shaders/grid/grid.rs:318-341). */
NXM_API int nxm_grid_read_headers(nxm_state* state, int32_t* out, uint32_t max_blocks);
/* Sorted particle ids with extras (GpuParticles::sorted_ids). */
NXM_API int nxm_grid_sorted_len(nxm_state* state, uint32_t* out);
NXM_API int nxm_grid_read_sorted_ids(nxm_state* state, uint32_t* out, uint32_t max_len);
/* Nodes after the last step's grid update, 4 floats per node (velocity xyz,
 * mass), 64 per block in header order (Node, grid.rs:401-421). */
NXM_API int nxm_grid_read_nodes(nxm_state* state, float* out, uint32_t max_blocks);

/* Runs only the sort (+ P2G when `with_p2g`) of the next step on the current
 * particles, leaving the grid readable; particles are not advanced. */
NXM_API int nxm_debug_sort(nxm_pipeline* pipeline, nxm_state* state, int with_p2g);
/* Test of the bounded waits on bulk copies: enqueues a kernel whose wait on a
 * copy barrier can never complete (no copy is issued) and runs out after
 * `limit` rounds, recording NXM_STATUS_COPY_TIMEOUT in the state's status word
 * (nxm_synchronize then returns NXM_E_CUDA until the status is cleared). */
NXM_API int nxm_debug_copy_wait_timeout(nxm_state* state, uint32_t limit);
/* Test of the error paths of host calls that allocate device memory (no
 * counterpart in the reference): with `after` >= 0, the after-th device
 * allocation the library makes from now on (0: the next one; any state)
 * fails once with NXM_E_OOM, as a full GPU would make it fail; -1 disarms.
 * A call that fails this way leaves its state as it was before the call. */
NXM_API int nxm_debug_fail_allocation(int64_t after);

/* ---- autotuner --------------------------------------------------------------
 * Launch shapes of one state's step.  No counterpart in the reference (its
 * dispatch sizes are fixed per shader). */
typedef struct nxm_tuning {
    uint32_t p2g_ctas_per_sm;   /* 1..3 */
    uint32_t g2p_ctas_per_sm;   /* 1..4 */
    uint32_t sort_ctas_per_sm;  /* 1, 2, 4, 8 or 16: the sort's particle passes */
    uint32_t grid_ctas_per_sm;  /* 1, 2, 4, 8 or 16: the grid update */
    uint32_t sort_batch;        /* 2, 4 or 8 passes of 32 particles a sort warp loads together */
    uint32_t range_min_fill;    /* below this many particles per block G2P runs one block per unit */
    uint32_t density;           /* table key: particles per primary block, rounded down to a power of two */
    uint32_t scenes;            /* table key: live scenes rounded up to a power of two (0: not batched) */
    float ms_before;            /* ms per step before tuning (0 when no trial ran) */
    float ms_after;             /* ms per step of the chosen shapes */
} nxm_tuning;

/* Times the state's own steps under candidate launch shapes (one knob at a
 * time, the others held; `trial_steps` timed steps per candidate after one
 * untimed step) and keeps the fastest; the state advances by every step
 * taken (about 15 x (trial_steps + 1)).  The decision is cached in a
 * process-wide table keyed by (density, scenes); with trial_steps = 0 the
 * call only applies the table's entry for this state's key, if there is one.
 * `out` (may be null) receives the decision and its key. */
NXM_API int nxm_state_autotune(nxm_state* state, uint32_t trial_steps, nxm_tuning* out);
NXM_API int nxm_state_get_tuning(const nxm_state* state, nxm_tuning* out);
/* Sets the launch shapes (values outside the ranges above: NXM_E_INVALID). */
NXM_API int nxm_state_set_tuning(nxm_state* state, const nxm_tuning* tuning);
/* The decision table: copies up to `max_entries` entries, returns how many exist. */
NXM_API uint32_t nxm_tuning_table(nxm_tuning* out, uint32_t max_entries);

/* ---- block sort without device allocation ----------------------------- */

/* Limits of nxm_sort_blocks_noalloc: active blocks its fixed tables hold,
 * and particles per call. */
#define NXM_NOALLOC_MAX_BLOCKS 16384u
#define NXM_NOALLOC_MAX_PARTICLES (1u << 26)

/* Block activation and particle sort for callers that may not allocate GPU
 * memory: a host program (a game engine, a simulation service) that reserves
 * all of its device memory once at start-up and forbids allocations inside
 * its frame loop, so that a frame can neither fail for lack of memory nor
 * stall while the allocator synchronizes the device, or a plugin running in
 * such a program that is handed device buffers but no allocator.  No
 * counterpart in the reference: nexus_mpm always sorts inside
 * MpmPipeline::step on state-owned buffers.
 *
 * Computes the same activation and primary ordering as the sort of nxm_step
 * (every particle's 2x2x2 block neighbourhood is active; each block's primary
 * particles are grouped by z-slab) without allocating anything (no cudaMalloc,
 * cudaFree or allocating library call): the grid tables live in one fixed
 * device array of the library (about 1.9 MB per GPU, held until the process
 * exits).  The caller passes device buffers:
 *   positions     n x 4 floats (x, y, z, unused), 16-byte aligned;
 *   sorted_ids    n uint32: particle ids grouped by primary block;
 *   block_vids    max_blocks x 4 int32 (16-byte aligned): block x, y, z and
 *                 packed key, in header order;
 *   block_ranges  max_blocks x 2 uint32 (8-byte aligned): first index into
 *                 sorted_ids and number of primary particles of each block
 *                 (0 for blocks that are only +1 neighbours).
 * `num_blocks` (host) receives the number of active blocks.  `stream` is a
 * cudaStream_t (NULL = legacy default stream); the call reads the result
 * back and waits for the stream before returning, so it blocks the host.
 *
 * Limits: more than min(max_blocks, NXM_NOALLOC_MAX_BLOCKS) active blocks
 * (including a scene whose blocks overflow the fixed hash) or more than
 * NXM_NOALLOC_MAX_PARTICLES particles return NXM_E_CAPACITY.
 * The first call on a device (with that device current) looks up the fixed
 * array's device address and keeps it for the life of the process; make that
 * first call before any stream capture, and do not use this entry point
 * across a cudaDeviceReset.  Every call reuses the same array and clears what
 * must start at zero, so calls whose GPU work overlaps (other streams or host
 * threads) race and must be serialized by the caller. */
NXM_API int nxm_sort_blocks_noalloc(const float* positions, uint32_t n, float cell_width, uint32_t* sorted_ids,
                                    int32_t* block_vids, uint32_t* block_ranges, uint32_t max_blocks,
                                    uint32_t* num_blocks, void* stream);

/* ---- batched scenes ----------------------------------------------------------
 * The batched form of the step: many independent scenes (same cell width,
 * dt and gravity) advance together, each nxm_step being one launch sequence
 * for all of them.  Scene s owns its own region of the block-key space (a
 * cube of `scene_blocks` blocks per axis); its particles keep scene-local
 * positions, so a scene steps exactly as it would alone, and its colliders
 * act on its own grid nodes only.  No counterpart call in the reference,
 * which steps one MpmState per pipeline call (src_mpm/pipeline.rs:385-526).
 *
 * Enable before adding any particle or collider (0 turns it off).  Particle
 * blocks must stay within local block coordinates [1 - M, S - M - 3] with
 * S = scene_blocks, M = S / 8 (a [0, 1]^3 scene fits S = 64 at dx = 1/128);
 * nxm_scene_add refuses particles outside with NXM_E_INVALID.  In scene
 * mode particles change only through the scene calls: the particle-level
 * append / remove / chunk calls return NXM_E_INVALID. */
NXM_API int nxm_state_enable_scenes(nxm_state* state, uint32_t scene_blocks);
/* Scene slots available (0 when scenes are off). */
NXM_API uint32_t nxm_scene_capacity(const nxm_state* state);
/* Adds a scene: its particles (appended as one contiguous id range) and up to
 * 16 colliders (triangles indexed within `tri_vertices`, as for
 * nxm_state_set_colliders).  Returns NXM_E_CAPACITY when every slot is taken. */
NXM_API int nxm_scene_add(nxm_state* state, const nxm_particles_soa* particles, uint32_t count,
                          const nxm_collider* colliders, uint32_t num_colliders, const float* tri_vertices,
                          uint32_t num_triangles, uint32_t* scene);
/* Removes scenes with their particles and colliders; the particle ids of the
 * remaining scenes shift down, keeping their order. */
NXM_API int nxm_scene_remove(nxm_state* state, const uint32_t* scenes, uint32_t count);
/* The particle-id range [first, first + count) of a live scene. */
NXM_API int nxm_scene_range(const nxm_state* state, uint32_t scene, uint32_t* first, uint32_t* count);
/* Kinematic driving of collider `index` of a scene (as nxm_state_set_collider_velocity). */
NXM_API int nxm_scene_set_collider_velocity(nxm_state* state, uint32_t scene, uint32_t index, const float linvel[3],
                                            const float angvel[3]);
/* Positions of particles [first, first + count) (3 floats each); synchronizes. */
NXM_API int nxm_read_positions_range(nxm_state* state, uint32_t first, uint32_t count, float* out);

/* ---- particle chunks (NexusState, src/state.rs:665-774) -------------------
 * A chunk is a handle on a set of particles appended together (and later
 * extended).  Removals swap-remove the chunk's slots (highest first) as
 * GpuParticles::swap_remove does, moving the records on the device in one
 * pass, and keep every particle's chunk ownership through the relocations. */
NXM_API int nxm_chunk_add(nxm_state* state, const nxm_particle* particles, uint32_t count, uint32_t* chunk);
NXM_API int nxm_chunk_extend(nxm_state* state, uint32_t chunk, const nxm_particle* particles, uint32_t count);
NXM_API int nxm_chunk_remove(nxm_state* state, uint32_t chunk);
/* Removes up to `count` of the chunk's particles (highest slots first); the
 * chunk is kept even when emptied.  `removed` (nullable) receives the number. */
NXM_API int nxm_chunk_remove_particles(nxm_state* state, uint32_t chunk, uint32_t count, uint32_t* removed);
NXM_API int nxm_chunk_len(const nxm_state* state, uint32_t chunk, uint32_t* len);
/* Owner chunk of each particle (0xFFFFFFFF: appended outside a chunk), len() entries. */
NXM_API int nxm_chunk_of_particles(const nxm_state* state, uint32_t* out);

/* WgTimestepBounds::compute_bounds (src_mpm/solver/timestep_bound.rs:24-46,
 * kernel src_mpm_shaders/solver/timestep_bound.rs:59-115): the CFL bound on dt
 * over the enabled particles, from each model's sound speed and the particle
 * velocity plus its APIC term.  Enqueued on the state's stream and read back
 * (synchronizes).  `*max_dt` = bits / 1e12 as the reference returns it;
 * `bits` (nullable) receives the fixed-point value (dt * 1e12) as u32, or
 * 0xFFFFFFFF when no particle is enabled. */
NXM_API int nxm_state_estimate_timestep_bound(nxm_state* state, float* max_dt, uint32_t* bits);

/* NexusPipeline::simulate's MPM part (src/pipeline.rs:75-87) with adaptive
 * substeps: the frame's dt (the simulation params' dt) is split into n
 * substeps, n = clamp(ceil(dt / CFL bound), min_substeps, max_substeps), the
 * bound taken as nxm_state_estimate_timestep_bound gives it at the start of
 * the frame (the reference runs a fixed count, state.rs:136-137, which
 * min_substeps = max_substeps reproduces); then write_substep_params(n) and n
 * steps.  Synchronizes once (the bound); `substeps` (nullable) receives n. */
NXM_API int nxm_simulate_frame(nxm_pipeline* pipeline, nxm_state* state, uint32_t min_substeps,
                               uint32_t max_substeps, uint32_t* substeps);

/* ---- synchronisation and status ------------------------------------------ */

NXM_API int nxm_synchronize(nxm_state* state);
/* Device status bits (NXM_STATUS_*); synchronizes.  `clear` resets them. */
NXM_API int nxm_state_status(nxm_state* state, uint32_t* bits, int clear);
/* Pipelined status read for a step loop: enqueues, after the work issued so
 * far, a one-thread kernel that stores the status word into mapped pinned
 * host memory (no copy engine between steps), and returns in `*bits` the
 * word the previous call enqueued (waiting only for that store, so the stream
 * never drains; 0 on the first call).  Each step's status reaches the host
 * one call late. */
NXM_API int nxm_state_status_pipelined(nxm_state* state, uint32_t* bits);
/* Non-blocking status poll for loops that keep many steps queued: when the
 * word posted by an earlier call has been stored (its store ran on the GPU),
 * returns it with *ready = 1 and posts a new one after the work issued so
 * far; otherwise returns *ready = 0 at once and posts nothing.  The host
 * never waits.  No counterpart in the reference (its step has no status). */
NXM_API int nxm_state_status_poll(nxm_state* state, uint32_t* bits, int* ready);
/* Tickets: nxm_state_fence marks the work queued on the state's stream so
 * far; nxm_state_ticket_done tells (without waiting) whether that work has
 * run, nxm_state_ticket_wait waits for it.  Tickets complete in the order
 * they were taken.  They stand for the futures of the reference's async
 * reads (below): done = the future is ready, wait = .await. */
NXM_API int nxm_state_fence(nxm_state* state, uint64_t* ticket);
NXM_API int nxm_state_ticket_done(nxm_state* state, uint64_t ticket, int* done);
NXM_API int nxm_state_ticket_wait(nxm_state* state, uint64_t ticket);
/* GpuParticles::read_positions (src_mpm/solver/particle.rs:634-648, an async
 * read) for the ids [first, first + count): positions into `out` (count x 3
 * floats) without waiting; `*ticket` completes when `out` holds them.  `out`
 * must stay valid until then; with pinned memory (nxm_host_alloc) the copy
 * queues behind the steps in flight, with pageable memory the call waits for
 * them. */
NXM_API int nxm_read_positions_range_async(nxm_state* state, uint32_t first, uint32_t count, float* out,
                                           uint64_t* ticket);
/* The device status word (NXM_STATUS_*) as of this point of the stream,
 * copied asynchronously into `out` (pinned host memory, see nxm_host_alloc);
 * valid once `*ticket` is done.  A serving loop takes one after each result
 * read, so that a result is only handed out when no step before it reported
 * a status bit.  No counterpart in the reference (its step has no status). */
NXM_API int nxm_state_read_status_async(nxm_state* state, uint32_t* out, uint64_t* ticket);
/* Pinned (page-locked) host memory for asynchronous reads and uploads. */
NXM_API int nxm_host_alloc(size_t bytes, void** out);
NXM_API void nxm_host_free(void* ptr);
NXM_API const char* nxm_error_string(int code);

/* The CUDA stream (cudaStream_t) every call on this state is ordered on,
 * so that a caller can record events or order its own work against it. */
NXM_API void* nxm_state_cuda_stream(const nxm_state* state);

/* Launches of this library's own kernels issued since the state was created
 * (each graph replay counts its kernel nodes). */
NXM_API uint64_t nxm_state_kernel_launches(const nxm_state* state);

#ifdef __cplusplus
}
#endif

#endif /* NEXUS_MPM_H */
