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
    const float4* tri;       // trimesh triangles: 3 float4 per triangle
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
};

struct LaunchCfg {
    int sm_count;
    uint32_t hash_capacity;  // host copy, sizes the reset grid
    uint32_t block_capacity;
    uint32_t particle_capacity;
};

// Number of kernels each launcher issues (for the launch counter).
struct StepLaunches {
    int sort;
    int p2g;
    int grid;
    int g2p;
};

namespace fast {
void launch_sort(const DevPtrs& P, const LaunchCfg& c, bool canonical, cudaStream_t s);
void launch_p2g(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s);
void launch_grid_update(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s);
void launch_g2p_update(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s);
void launch_colliders_begin(const DevPtrs& P, cudaStream_t s);
void launch_colliders_end(const DevPtrs& P, cudaStream_t s);
}  // namespace fast

namespace exact {
void launch_p2g_gather(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s);
void launch_grid_update(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s);
void launch_g2p_update(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s);
}  // namespace exact

// Kernels issued per phase (sort counts the canonical segment sort when on).
int sort_launches(bool canonical);
constexpr int kP2gLaunches = 1;
constexpr int kGridLaunches = 1;
constexpr int kG2pLaunches = 1;
constexpr int kColliderLaunches = 2;

}  // namespace nxm
