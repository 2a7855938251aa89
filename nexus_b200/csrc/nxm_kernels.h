// Kernel launchers of one MPM step (host-visible declarations).
#pragma once

#include <cuda_runtime.h>

#include "nxm_layout.h"

namespace nxm {

// Device pointers of one state, passed by value to every kernel.
struct DevPtrs {
    PKin* kin;
    PDef* def;
    float4* pstate;          // model state words (plastic models)
    const Material* materials;
    DevCollider* colliders;
    const DevTri* tris;      // trimesh triangles of all trimesh colliders
    const DevBvhNode* bvh;   // their BVHs
    const Params* params;
    Counters* counters;
    // hash map of block keys
    uint32_t* hkey;
    uint32_t* hval;
    // block headers (struct of arrays)
    int4* bvid;              // x, y, z, packed key
    uint32_t* first;
    uint32_t* nprim;
    uint32_t* nwx;           // num_particles_with_extras
    uint32_t* cursors;       // NUM_BUCKETS per block
    uint32_t* nbh;           // NUM_NBH per block
    float4* nodes;           // 64 per block
    uint32_t* sorted;        // sorted ids with extras
    uint2* pcode;            // per particle: packed block key, assoc code (ax | ay<<2 | az<<4)
    uint32_t* phdr;          // per particle: primary header id
    uint32_t* scan_tmp;      // per block: offset inside its scan tile
    uint32_t* tile_sums;     // per scan tile of kScanTile blocks: its total
    // per run of kRangeChunk sorted positions: the block holding its first
    // position (written by the scan; the fast G2P walks the sorted list in
    // these runs)
    uint32_t* chunk_blk;
    uint32_t chunk_cap;
    // G2P output.  In place: the *_out pointers equal the inputs and pid_in is
    // null.  Reordering: sorted entry j is written to slot j of the *_out
    // records, pid_out[j] = pid_in[its source slot] (pid = particle id).
    PKin* kin_out;
    PDef* def_out;
    float4* pstate_out;
    const uint32_t* pid_in;
    uint32_t* pid_out;
    // batched scenes: scene of each particle id, and each scene's colliders
    // [x, x + y) in `colliders`
    const uint32_t* pscene;
    const uint2* scene_cols;
    // CPIC: node distance field (distance bits, affinity + sign bits, closest
    // collider, unused), the nodes' incompatible momentum / velocity + mass,
    // and per particle id 3 float4: normal + signed distance, rigid velocity
    // + affinity bits, and the properties the step does not move (boundary
    // friction, then the render-only init radius, phase, group id bits).
    uint4* ncdf;
    float4* nodes_inc;
    float4* pcdf;
    // CPIC rigid particles of the trimesh colliders: local and world
    // position (w = packed triangle / collider word), block-activation flag,
    // per block the count (then the placement cursor) and first entry of the
    // block-sorted list (own block plus extras).
    uint32_t nrp;
    const float4* rp_local;
    float4* rp_world;
    uint8_t* rp_need;
    uint32_t* rp_count;
    uint32_t* rp_first;
    uint32_t* rp_sorted;
};

constexpr uint32_t kScanTile = 256;  // blocks per scan tile (one per thread of a scan CTA)
constexpr uint32_t kRangeChunk = 256;  // sorted positions per fast-G2P run (one per thread of its CTA)

// Launch shapes the autotuner picks per state (nxm_state_autotune); the
// defaults are the hand-measured best of the 2 M-particle sand + water scene.
struct Tuning {
    uint32_t p2g_ctas = 3;    // P2G CTAs per SM (its launch bounds fit 3)
    uint32_t g2p_ctas = 4;    // G2P CTAs per SM (its launch bounds fit 4)
    uint32_t sort_ctas = 8;   // CTAs per SM of the sort's particle passes
    uint32_t grid_ctas = 8;   // grid update CTAs per SM
    uint32_t sort_batch = 4;  // 2, 4 or 8 passes of 32 particles a sort warp loads together
};

struct LaunchCfg {
    int sm_count;
    uint32_t hash_capacity;  // host copy, sizes the reset grid
    uint32_t block_capacity;
    uint32_t particle_capacity;
    Tuning t;
};

// Number of kernels each launcher issues (for the launch counter).
struct StepLaunches {
    int sort;
    int p2g;
    int grid;
    int g2p;
};

namespace fast {
// `with_extras`: also list every particle as an "extra" in the +1 neighbour
// blocks its stencil reaches (the reference's full sorted-id layout, used by
// the gather-form P2G); the scatter P2G needs the primaries only.
// `canonical`: order each bucket by ascending particle id.
// `rigid`: also activate the blocks of the CPIC rigid particles and sort them
// by block (P.nrp > 0; their world positions already written).
void launch_sort(const DevPtrs& P, const LaunchCfg& c, bool with_extras, bool canonical, cudaStream_t s,
                 bool rigid = false);
constexpr int kRigidSortLaunches = 5;
void launch_p2g(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s);
void launch_grid_update(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s);
int launch_g2p_update(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s);  // returns the kernels issued
// CPIC scatter P2G (compatible and incompatible fields; particles in id order).
void launch_p2g_cpic(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s);
// A bulk-copy barrier wait that runs out after `limit` rounds (test of the
// timeout path: records STATUS_COPY_TIMEOUT).
void launch_copy_wait_timeout(Counters* counters, uint32_t limit, cudaStream_t s);
}  // namespace fast

// Fast-arithmetic CPIC grid update and per-block G2P (nxm_transfer_fast_cpic.cu).
namespace fast_cpic {
void launch_grid_update(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s);
int launch_g2p_update(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s);
}  // namespace fast_cpic

namespace exact {
void launch_p2g_gather(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s);
// Min over particles of the CFL bound into counters->dt_bound (reset by the caller).
void launch_timestep_bound(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s);
// CPIC distance fields: per node (analytic colliders), then per particle.
void launch_grid_update_cdf(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s);
void launch_g2p_cdf(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s);
// CPIC rigid particles: world positions from the collider poses, and the
// triangle projections merged into the node distance field.
void launch_rigid_transform(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s);
void launch_p2g_cdf(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s);
void launch_grid_update(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s);
int launch_g2p_update(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s);  // returns the kernels issued
}  // namespace exact

// Render data (prep_readback.rs): the particle records, the slot -> id map of
// block-ordered storage (null: slot = id), the render mode and palette.
enum : uint32_t {
    RENDER_DEFAULT = 0,
    RENDER_VOLUME = 1,
    RENDER_VELOCITY = 2,
    RENDER_PHASE = 3,
    RENDER_CDF_NORMALS = 4,
    RENDER_CDF_DISTANCES = 5,
    RENDER_CDF_SIGNS = 6,
};
struct RenderSrc {
    const PKin* kin;
    const PDef* def;
    const float4* pcdf;  // per id: normal + signed distance, rigid velocity + affinity, render properties
    const uint32_t* pid;
    uint32_t n;
    uint32_t mode;
    const float4* palette;
    uint32_t num_groups;
    float dx, dt;
    int sm_count;
};
void launch_prep_readback(const RenderSrc& in, float4* out, cudaStream_t s);
void launch_prep_render(const RenderSrc& in, float* positions, float* deformations, float* colors, cudaStream_t s);
void launch_prep_readback_rigid(const RenderSrc& in, const float4* world, uint32_t nrp, const float4* colors,
                                float4* out, cudaStream_t s);

// Primary-only block sort of plain float4 positions (x, y, z, unused): no
// per-particle scratch; P.sorted receives the ids, P.nodes may be null.
void launch_sort_positions(const DevPtrs& P, const LaunchCfg& c, const float4* pos, cudaStream_t s);
constexpr int kSortPositionsLaunches = 8;

// Kernels issued per phase (sort counts the canonical segment sort when on).
int sort_launches(bool canonical);
constexpr int kP2gLaunches = 1;
constexpr int kGridLaunches = 1;

}  // namespace nxm
