// Host side of the library: MpmState / MpmPipeline equivalents behind the C
// ABI of include/nexus_mpm.h (src_mpm/pipeline.rs, src_mpm/solver/particle.rs,
// src_mpm/grid/grid.rs).
//
// A state owns its device buffers and one CUDA stream.  The step's kernels
// read every size and parameter from device memory (Params, Counters) and
// loop grid-stride over device-side counts, so the whole step is captured
// once as a CUDA graph and replayed; the graph is rebuilt only when a
// buffer is reallocated or the mode changes.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <initializer_list>
#include <map>
#include <mutex>
#include <new>
#include <set>
#include <thread>
#include <deque>
#include <vector>

#include "../../include/nexus_mpm.h"
#include "nxm_kernels.h"
#include "nxm_layout.h"

using namespace nxm;

namespace {

uint32_t next_pow2(uint32_t v) {
    uint32_t c = 1;
    while (c < v && c < 0x80000000u) c <<= 1;
    return c;
}

#define NXM_TRY(expr)                                   \
    do {                                                \
        cudaError_t e_ = (expr);                        \
        if (e_ != cudaSuccess) {                        \
            (void)cudaGetLastError();                   \
            return e_ == cudaErrorMemoryAllocation ? NXM_E_OOM : NXM_E_CUDA; \
        }                                               \
    } while (0)
// Propagates a nonzero NXM_* result.
#define NXM_TRY_RC(expr)        \
    do {                        \
        const int rc_ = (expr); \
        if (rc_) return rc_;    \
    } while (0)

// Host-side fault injection (nxm_debug_fail_allocation): armed with k >= 0,
// the k-th device allocation from then on (0: the next one) reports
// cudaErrorMemoryAllocation once and the hook disarms; -1: off.  Counts the
// library's own cudaMalloc and pool allocations, every state alike.
std::atomic<int64_t> g_alloc_fail_in{-1};

bool injected_alloc_failure() {
    int64_t v = g_alloc_fail_in.load();
    while (v >= 0)
        if (g_alloc_fail_in.compare_exchange_weak(v, v - 1)) return v == 0;
    return false;
}

template <class T>
cudaError_t dalloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    if (injected_alloc_failure()) return cudaErrorMemoryAllocation;
    return cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T));
}
template <class T>
void dfree(T*& p) {
    if (p) cudaFree(p);
    p = nullptr;
}

// Runs of kRangeChunk sorted positions a state of `cap` particles needs
// (the fast path lists each particle once).
uint32_t chunk_cap_for(uint32_t cap) { return cap / kRangeChunk + 2; }

float bits_f(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
uint32_t f_bits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

bool model_has_state(uint32_t tag) {
    return tag == MODEL_SAND_LINEAR || tag == MODEL_SAND_NEO_HOOKEAN || tag == MODEL_SNOW;
}
int model_state_words(uint32_t tag) {
    if (tag == MODEL_SAND_LINEAR || tag == MODEL_SAND_NEO_HOOKEAN) return 3;
    if (tag == MODEL_SNOW) return 1;
    return 0;
}

// Packs selected 4-byte fields of the records of particles [first, first + n)
// into a dense array.
__global__ void k_pack_fields(const uint32_t* __restrict__ src, uint32_t stride_words, uint32_t first, uint32_t n,
                              const int* __restrict__ offsets, int nfields, uint32_t* __restrict__ dst) {
    const uint32_t total = n * (uint32_t)nfields;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const uint32_t p = first + t / (uint32_t)nfields, f = t % (uint32_t)nfields;
        dst[t] = src[(size_t)p * stride_words + offsets[f]];
    }
}

// Permuted storage (slot p holds particle pid[p]): scatter the fields of the
// particles with id in [first, first + count) by id (all n slots are scanned).
__global__ void k_pack_fields_perm(const uint32_t* __restrict__ src, uint32_t stride_words, uint32_t n,
                                   uint32_t first, uint32_t count, const int* __restrict__ offsets, int nfields,
                                   const uint32_t* __restrict__ pid, uint32_t* __restrict__ dst) {
    const uint32_t total = n * (uint32_t)nfields;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const uint32_t p = t / (uint32_t)nfields, f = t % (uint32_t)nfields;
        const uint32_t id = pid[p] - first;
        if (id < count) dst[(size_t)id * nfields + f] = src[(size_t)p * stride_words + offsets[f]];
    }
}

// ---- stable removal of particle-id ranges (compaction over storage slots) ----
// `ranges` sorted and disjoint, `cum[i]` = total length of ranges before i.
// Tiles of 1024 slots; 256 threads x 4 slots.
__device__ __forceinline__ uint32_t range_of(uint32_t id, const uint2* __restrict__ ranges, uint32_t nr) {
    uint32_t lo = 0, hi = nr;  // first range with start > id
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (ranges[mid].x <= id) lo = mid + 1; else hi = mid;
    }
    return lo;  // ranges[lo - 1] is the last one starting at or before id
}
__device__ __forceinline__ bool removed_id(uint32_t id, const uint2* __restrict__ ranges, uint32_t nr) {
    const uint32_t r = range_of(id, ranges, nr);
    return r > 0 && id < ranges[r - 1].y;
}
__device__ __forceinline__ uint32_t new_id_of(uint32_t id, const uint2* __restrict__ ranges,
                                              const uint32_t* __restrict__ cum, uint32_t nr) {
    const uint32_t r = range_of(id, ranges, nr);
    return r == 0 ? id : id - cum[r - 1] - (ranges[r - 1].y - ranges[r - 1].x);  // id is past range r - 1
}
__device__ __forceinline__ uint32_t survivors4(uint32_t base, uint32_t n, const uint32_t* __restrict__ pid,
                                              const uint2* __restrict__ ranges, uint32_t nr, bool keep[4]) {
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t p = base + k;
        keep[k] = p < n && !removed_id(pid ? pid[p] : p, ranges, nr);
        c += keep[k] ? 1u : 0u;
    }
    return c;
}
__device__ __forceinline__ uint32_t block_excl_scan256(uint32_t v, uint32_t* sh, uint32_t* total) {
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= (uint32_t)o) incl += y;
    }
    if (lane == 31) sh[w] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int i = 0; i < 8; ++i) {
            const uint32_t t = sh[i];
            sh[i] = run;
            run += t;
        }
        sh[8] = run;
    }
    __syncthreads();
    const uint32_t out = sh[w] + incl - v;
    *total = sh[8];
    __syncthreads();
    return out;
}
__global__ void __launch_bounds__(256) k_rm_count(uint32_t n, const uint32_t* __restrict__ pid,
                                                  const uint2* __restrict__ ranges, uint32_t nr,
                                                  uint32_t* __restrict__ tiles) {
    __shared__ uint32_t sh[9];
    bool keep[4];
    const uint32_t c = survivors4(blockIdx.x * 1024u + threadIdx.x * 4u, n, pid, ranges, nr, keep);
    uint32_t total;
    block_excl_scan256(c, sh, &total);
    if (threadIdx.x == 0) tiles[blockIdx.x] = total;
}
__global__ void __launch_bounds__(1024) k_rm_scan(uint32_t* __restrict__ tiles, uint32_t ntiles) {
    __shared__ uint32_t carry;
    __shared__ uint32_t wsum[32];
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < ntiles; base += 1024u) {
        const uint32_t i = base + threadIdx.x;
        const uint32_t v = i < ntiles ? tiles[i] : 0u;
        const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
        uint32_t incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= (uint32_t)o) incl += y;
        }
        if (lane == 31) wsum[w] = incl;
        __syncthreads();
        if (w == 0) {
            const uint32_t s = wsum[lane];
            uint32_t si = s;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, si, o);
                if (lane >= (uint32_t)o) si += y;
            }
            wsum[lane] = si - s;
        }
        __syncthreads();
        if (i < ntiles) tiles[i] = carry + wsum[w] + incl - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry += wsum[31] + incl;
        __syncthreads();
    }
}
__global__ void __launch_bounds__(256) k_rm_move(uint32_t n, const PKin* __restrict__ kin, const PDef* __restrict__ def,
                                                 const float4* __restrict__ pstate, const uint32_t* __restrict__ pid,
                                                 const uint2* __restrict__ ranges, const uint32_t* __restrict__ cum,
                                                 uint32_t nr, const uint32_t* __restrict__ tiles,
                                                 PKin* __restrict__ kin_to, PDef* __restrict__ def_to,
                                                 float4* __restrict__ pstate_to, uint32_t* __restrict__ pid_to) {
    __shared__ uint32_t sh[9];
    bool keep[4];
    const uint32_t base = blockIdx.x * 1024u + threadIdx.x * 4u;
    const uint32_t c = survivors4(base, n, pid, ranges, nr, keep);
    uint32_t total;
    uint32_t dst = tiles[blockIdx.x] + block_excl_scan256(c, sh, &total);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (!keep[k]) continue;
        const uint32_t p = base + k;
        kin_to[dst] = kin[p];
        def_to[dst] = def[p];
        pstate_to[dst] = pstate[p];
        if (pid) pid_to[dst] = new_id_of(pid[p], ranges, cum, nr);
        ++dst;
    }
}

// Id-indexed arrays (K elements per id) follow a range removal: entry id goes to its new id.
template <class T, int K>
__global__ void k_rm_ids(uint32_t n, const T* __restrict__ src, const uint2* __restrict__ ranges,
                         const uint32_t* __restrict__ cum, uint32_t nr, T* __restrict__ dst) {
    for (uint32_t id = blockIdx.x * blockDim.x + threadIdx.x; id < n; id += gridDim.x * blockDim.x)
        if (!removed_id(id, ranges, nr)) {
            const uint32_t to = new_id_of(id, ranges, cum, nr);
#pragma unroll
            for (int k = 0; k < K; ++k) dst[(size_t)K * to + k] = src[(size_t)K * id + k];
        }
}

// Swap-removal data movement: record pairs[i].y moves to slot pairs[i].x.
// Every source is at or above the new length and every destination below it,
// so the moves are independent.
__global__ void k_move_records(PKin* __restrict__ kin, PDef* __restrict__ def, float4* __restrict__ pstate,
                               float4* __restrict__ pcdf, const uint2* __restrict__ pairs, uint32_t count) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const uint2 m = pairs[i];
        kin[m.x] = kin[m.y];
        def[m.x] = def[m.y];
        pstate[m.x] = pstate[m.y];
#pragma unroll
        for (int k = 0; k < 3; ++k) pcdf[3u * m.x + k] = pcdf[3u * m.y + k];
    }
}

// Kinematic driving of many colliders: vel6[i] = linvel xyz, angvel xyz of collider first + i.
__global__ void k_set_velocities(DevCollider* __restrict__ cols, const float* __restrict__ vel6, uint32_t first,
                                 uint32_t count) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        DevCollider& c = cols[first + i];
        const float* v = vel6 + 6 * (size_t)i;
        c.linvel[0] = v[0]; c.linvel[1] = v[1]; c.linvel[2] = v[2];
        c.angvel[0] = v[3]; c.angvel[1] = v[4]; c.angvel[2] = v[5];
    }
}

// One collider's velocity, passed by value (no host staging, no stream sync).
struct Vel6 {
    float v[6];
};
__global__ void k_set_velocity(DevCollider* __restrict__ cols, uint32_t index, Vel6 vel) {
    if (threadIdx.x == 0) {
        DevCollider& c = cols[index];
        c.linvel[0] = vel.v[0]; c.linvel[1] = vel.v[1]; c.linvel[2] = vel.v[2];
        c.angvel[0] = vel.v[3]; c.angvel[1] = vel.v[4]; c.angvel[2] = vel.v[5];
    }
}

__global__ void k_fill(uint32_t* __restrict__ out, uint32_t value, uint32_t count) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) out[t] = value;
}

// The status word stored straight into mapped pinned host memory: no copy
// engine between two steps (a 4-byte device-to-host copy costs tens of
// microseconds of stream time there).
__global__ void k_post_status(const Counters* __restrict__ c, volatile uint32_t* out) {
    if (threadIdx.x == 0) {
        *out = c->status;
        __threadfence_system();
    }
}

__global__ void k_iota(uint32_t* __restrict__ out, uint32_t first, uint32_t count) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) out[t] = first + t;
}

// Back to id order: record of slot p goes to slot pid[p] of the other buffers.
__global__ void k_unpermute(const PKin* __restrict__ kin, const PDef* __restrict__ def,
                            const float4* __restrict__ pstate, const uint32_t* __restrict__ pid, uint32_t n,
                            PKin* __restrict__ kin_to, PDef* __restrict__ def_to, float4* __restrict__ pstate_to) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const uint32_t id = pid[p];
        kin_to[id] = kin[p];
        def_to[id] = def[p];
        pstate_to[id] = pstate[p];
    }
}

}  // namespace

struct nxm_pipeline {
    int device = 0;
    int sm_count = 0;
};

struct nxm_state {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;

    // parameters
    float base_dt = 1.0f / 60.0f;
    float gravity[3] = {0.f, 0.f, 0.f};
    float dt = 1.0f / 60.0f;
    float dx = 1.0f;
    bool use_cpic = false;
    bool deterministic = false;

    // particles.  Fast mode keeps the records in the previous step's sorted
    // order: each step's G2P writes them to the *_alt buffers, which then
    // become current (`parity` counts the swaps mod 2); pid[slot] is the
    // particle id of a slot while `permuted`, otherwise slot == id.
    uint32_t n = 0, pcap = 0;
    char* pslab = nullptr;  // the one allocation the per-particle arrays below are carved from
    PKin* kin = nullptr;
    PDef* def = nullptr;
    float4* pstate = nullptr;
    PKin* kin_alt = nullptr;
    PDef* def_alt = nullptr;
    float4* pstate_alt = nullptr;
    uint32_t* pid = nullptr;
    uint32_t* pid_alt = nullptr;
    bool permuted = false;
    int parity = 0;
    const uint32_t* sort_pid = nullptr;  // slot -> id map of the storage the last sort ran on (null: identity)
    uint2* pcode = nullptr;
    uint32_t* phdr = nullptr;
    uint32_t* sorted = nullptr;
    // particle chunks (src/state.rs:665-774): owner chunk of each particle id
    // (NONE for particles appended outside a chunk) and the live chunks' sizes
    std::vector<uint32_t> slot2chunk;  // empty until the first chunk is created
    bool chunks_used = false;
    std::map<uint32_t, uint32_t> chunks;
    uint32_t next_chunk = 0;

    // materials (deduplicated model words)
    std::vector<Material> materials;
    std::map<std::vector<uint32_t>, uint32_t> material_index;
    Material* d_materials = nullptr;
    uint32_t mat_cap = 0;
    bool materials_dirty = false;

    // grid
    uint32_t block_cap = 0, hash_cap = 0;
    char* gslab = nullptr;  // the one allocation the grid arrays below are carved from
    uint32_t* hkey = nullptr;
    uint32_t* hval = nullptr;
    int4* bvid = nullptr;
    uint32_t *first = nullptr, *nprim = nullptr, *nwx = nullptr, *cursors = nullptr, *nbh = nullptr;
    float4* nodes = nullptr;
    uint32_t* scan_tmp = nullptr;
    uint32_t* tile_sums = nullptr;

    // colliders
    std::vector<DevCollider> colliders;
    DevCollider* d_colliders = nullptr;
    uint32_t col_cap = 0;
    // bulk collider velocities: pinned host slots (a ring, each reused only
    // after the copy issued from it has run) and their device copies
    static constexpr int kVelSlots = 4;
    float* d_vel6 = nullptr;
    float* h_vel6 = nullptr;
    cudaEvent_t vel_done[kVelSlots] = {};
    size_t vel_cap = 0;  // floats per slot
    int vel_slot = 0;
    // pipelined status reads: pinned words and their copy events
    uint32_t* h_status = nullptr;    // two mapped pinned words (host view)
    uint32_t* h_status_dev = nullptr;  // the same words, device view
    cudaEvent_t status_done[2] = {};
    uint64_t status_calls = 0;
    // nxm_state_status_poll: its own posted word (slot 0 of h_poll), the
    // event after that post, and whether a post is outstanding
    uint32_t* h_poll = nullptr;
    uint32_t* h_poll_dev = nullptr;
    cudaEvent_t poll_done = nullptr;
    bool poll_outstanding = false;

    // launch shapes (nxm_state_autotune); range_min_fill goes to Params
    Tuning tuning;
    uint32_t range_min_fill = 64;

    // batched scenes (scene_blocks != 0): scene slots on the block-key grid
    // (see Params), each a contiguous range of particle ids with its own colliders
    struct Scene {
        bool live = false;
        uint32_t first = 0, count = 0;
        std::vector<nxm_collider> cols;
        std::vector<float> tri;
    };
    uint32_t scene_blocks = 0;
    int scene_margin = 0;
    int scene_cmin[3] = {0, 0, 0};
    uint32_t scene_cells[3] = {0, 0, 0};
    std::vector<Scene> scenes;
    uint32_t* d_pscene = nullptr;       // scene of each particle id (device)
    float4* d_pcdf = nullptr;           // CPIC particle fields, 3 float4 per particle id
    float4* d_pcdf_alt = nullptr;
    uint4* d_ncdf = nullptr;            // CPIC node distance fields (allocated with CPIC on)
    float4* d_nodes_inc = nullptr;      // CPIC incompatible node fields
    uint32_t* d_pscene_alt = nullptr;
    uint2* d_scene_cols = nullptr;      // per scene slot: its colliders in the table
    uint32_t* d_tiles = nullptr;        // compaction scratch, one word per 1024 particles
    uint32_t* d_chunk_blk = nullptr;    // block of each run of kRangeChunk sorted positions
    DevTri* d_tris = nullptr;       // triangles of every trimesh collider (one copy per collider)
    DevBvhNode* d_bvh = nullptr;    // their BVHs
    std::vector<DevTri> tris_host;  // host copy of d_tris
    std::vector<uint32_t> tri_base; // per collider: its first record in d_tris (trimesh only)

    // CPIC rigid particles: surface samples of the trimesh colliders
    // (local position + packed triangle / collider word), their world
    // positions, activation flags and block-sorted list; per block counts
    // and first entries (sized by the grid capacity, with the CPIC node fields)
    uint32_t nrp = 0;
    std::vector<float4> rp_host;
    float4* d_rp_local = nullptr;
    float4* d_rp_world = nullptr;
    uint8_t* d_rp_need = nullptr;
    uint32_t* d_rp_sorted = nullptr;
    uint32_t* d_rp_count = nullptr;
    uint32_t* d_rp_first = nullptr;

    // control
    Params* d_params = nullptr;
    Counters* d_counters = nullptr;
    Counters* h_counters = nullptr;  // pinned
    bool params_dirty = true;

    // graphs (one per buffer parity)
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    bool graph_valid[2] = {false, false};
    int graph_kernels = 0;
    uint64_t launches = 0;

    // render data (prep_readback): record scratch and palette
    float4* d_render = nullptr;
    size_t render_cap = 0;  // float4s
    float4* d_palette = nullptr;
    uint32_t palette_cap = 0;

    // pinned staging ring for host -> device copies (see upload_async)
    struct StagingSpan {
        size_t begin, end;
        cudaEvent_t done;
    };
    char* stg = nullptr;
    size_t stg_cap = 0, stg_head = 0;
    std::deque<StagingSpan> stg_live;
    // outgrown rings, each with an event recorded after the last copy out of
    // it; freed once that event has completed (see free_retired_rings)
    struct RetiredRing {
        char* ring;
        cudaEvent_t done;
    };
    std::vector<RetiredRing> stg_retired;
    std::vector<cudaEvent_t> event_pool;

    // scratch of uploads, removals and reads: a memory pool of this state that
    // keeps what it has grown to (the device's default pool hands memory back
    // at every synchronisation, so each upload would map its scratch anew)
    cudaMemPool_t pool = nullptr;

    // stream-ordered tickets (nxm_state_fence): the events of tickets not yet
    // known complete, oldest first; tickets up to done_ticket are complete
    std::deque<std::pair<uint64_t, cudaEvent_t>> fences;
    uint64_t next_ticket = 1, done_ticket = 0;

    // scratch for readback packing
    uint32_t* d_pack = nullptr;
    size_t pack_cap = 0;
    int* d_offsets = nullptr;
};

namespace {

// Fast mode keeps the records in block order; the deterministic and CPIC
// steps work in place, in id order (CPIC's per-particle fields are id-indexed).
bool reorders(const nxm_state* s) { return !s->deterministic && !s->use_cpic; }

DevPtrs dev_ptrs(nxm_state* s) {
    DevPtrs P{};
    P.kin = s->kin;
    P.def = s->def;
    P.pstate = s->pstate;
    if (reorders(s)) {
        P.kin_out = s->kin_alt;
        P.def_out = s->def_alt;
        P.pstate_out = s->pstate_alt;
        P.pid_in = s->pid;
        P.pid_out = s->pid_alt;
    } else {
        P.kin_out = s->kin;
        P.def_out = s->def;
        P.pstate_out = s->pstate;
        P.pid_in = nullptr;
        P.pid_out = nullptr;
    }
    P.materials = s->d_materials;
    P.colliders = s->d_colliders;
    P.pscene = s->d_pscene;
    P.ncdf = s->d_ncdf;
    P.nodes_inc = s->d_nodes_inc;
    P.pcdf = s->d_pcdf;
    P.scene_cols = s->d_scene_cols;
    P.tris = s->d_tris;
    P.bvh = s->d_bvh;
    if (s->use_cpic && s->nrp) {
        P.nrp = s->nrp;
        P.rp_local = s->d_rp_local;
        P.rp_world = s->d_rp_world;
        P.rp_need = s->d_rp_need;
        P.rp_sorted = s->d_rp_sorted;
        P.rp_count = s->d_rp_count;
        P.rp_first = s->d_rp_first;
    }
    P.params = s->d_params;
    P.counters = s->d_counters;
    P.hkey = s->hkey;
    P.hval = s->hval;
    P.bvid = s->bvid;
    P.first = s->first;
    P.nprim = s->nprim;
    P.nwx = s->nwx;
    P.cursors = s->cursors;
    P.nbh = s->nbh;
    P.nodes = s->nodes;
    P.sorted = s->sorted;
    P.pcode = s->pcode;
    P.phdr = s->phdr;
    P.scan_tmp = s->scan_tmp;
    P.tile_sums = s->tile_sums;
    P.chunk_blk = s->d_chunk_blk;
    P.chunk_cap = chunk_cap_for(s->pcap);
    return P;
}

LaunchCfg launch_cfg(nxm_state* s) {
    LaunchCfg c{};
    c.sm_count = s->sm_count;
    c.hash_capacity = s->hash_cap;
    c.block_capacity = s->block_cap;
    c.particle_capacity = s->pcap;
    c.t = s->tuning;
    return c;
}

// ---- pinned staging -------------------------------------------------------------
//
// Host data bound for the device is copied into a ring of pinned memory and
// sent from there with cudaMemcpyAsync, so the copy is ordered on the stream
// behind the queued work without the host waiting for it (a copy from
// pageable memory would first drain the stream).  An event recorded after
// each copy marks when its ring region may be written again.

// Stream-ordered scratch from the state's pool (freed with cudaFreeAsync).
template <class T>
cudaError_t scratch_alloc(nxm_state* s, T** p, size_t bytes) {
    *p = nullptr;
    if (injected_alloc_failure()) return cudaErrorMemoryAllocation;
    return cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), bytes, s->pool, s->stream);
}

cudaError_t take_event(nxm_state* s, cudaEvent_t* e) {
    if (!s->event_pool.empty()) {
        *e = s->event_pool.back();
        s->event_pool.pop_back();
        return cudaSuccess;
    }
    return cudaEventCreateWithFlags(e, cudaEventDisableTiming);
}

// Frees the outgrown staging rings whose copies have all run (the event
// recorded when the ring was retired has completed).  `drained`: the caller
// has just waited for the stream, so every such event is complete.
// cudaFreeHost may wait for the device, so calls that must not block (the
// ring reservation of a queued upload) free only while the stream is idle;
// ticket waits and nxm_synchronize free as soon as the copies are done.
// A serving loop that only waits on tickets therefore keeps no outgrown ring
// past the first ticket wait after its copies ran.
void free_retired_rings(nxm_state* s, bool drained = true) {
    size_t kept = 0;
    for (auto& r : s->stg_retired) {
        const bool done = drained || cudaEventQuery(r.done) == cudaSuccess;
        if (done) {
            cudaFreeHost(r.ring);
            s->event_pool.push_back(r.done);
        } else {
            s->stg_retired[kept++] = r;
        }
    }
    s->stg_retired.resize(kept);
    (void)cudaGetLastError();  // a not-ready query is not an error
}

// A new ring of at least `bytes` * 4 (twice the old one, 1 MB at least, up
// to kRingMax).  The old ring is kept, not freed, until the stream drains:
// its copies may still be queued behind other work, and the host does not
// wait for them here.
constexpr size_t kRingMax = size_t(1) << 30;
cudaError_t staging_grow(nxm_state* s, size_t bytes) {
    for (const auto& sp : s->stg_live) s->event_pool.push_back(sp.done);  // an event may be recorded again
    s->stg_live.clear();
    if (s->stg) {
        cudaEvent_t done;
        cudaError_t e = take_event(s, &done);
        if (e == cudaSuccess) e = cudaEventRecord(done, s->stream);  // after the last copy out of the ring
        if (e != cudaSuccess) return e;
        s->stg_retired.push_back(nxm_state::RetiredRing{s->stg, done});
    }
    s->stg = nullptr;
    const size_t cap = std::max({bytes * 4, std::min(s->stg_cap * 2, kRingMax), size_t(1) << 20});
    s->stg_cap = 0;
    s->stg_head = 0;
    const cudaError_t e = cudaMallocHost(reinterpret_cast<void**>(&s->stg), cap);
    if (e != cudaSuccess) {
        s->stg = nullptr;
        return e;
    }
    s->stg_cap = cap;
    return cudaSuccess;
}

// A ring region of `bytes` (256-aligned) whose earlier copies have run.
cudaError_t staging_reserve(nxm_state* s, size_t bytes, char** out) {
    bytes = (bytes + 255) & ~size_t(255);
    if (!s->stg_retired.empty() && cudaStreamQuery(s->stream) == cudaSuccess) free_retired_rings(s);
    (void)cudaGetLastError();
    if (bytes * 2 > s->stg_cap) {
        const cudaError_t e = staging_grow(s, bytes);
        if (e != cudaSuccess) return e;
    }
    if (s->stg_head + bytes > s->stg_cap) s->stg_head = 0;
    size_t lo = s->stg_head, hi = lo + bytes;
    int newest = -1;  // copies complete in stream order: waiting for the newest overlap covers the older
    for (size_t i = 0; i < s->stg_live.size(); ++i)
        if (s->stg_live[i].begin < hi && lo < s->stg_live[i].end) newest = (int)i;
    if (newest >= 0 && s->stg_cap < kRingMax && cudaEventQuery(s->stg_live[newest].done) == cudaErrorNotReady) {
        // that region is still queued behind other work: a larger ring instead of a wait
        const cudaError_t e = staging_grow(s, bytes);
        if (e != cudaSuccess) return e;
        lo = 0;
        hi = bytes;
        newest = -1;
    }
    if (newest >= 0) {
        cudaError_t e = cudaEventSynchronize(s->stg_live[newest].done);
        if (e != cudaSuccess) return e;
        for (int i = 0; i <= newest; ++i) s->event_pool.push_back(s->stg_live[i].done);
        s->stg_live.erase(s->stg_live.begin(), s->stg_live.begin() + newest + 1);
    }
    *out = s->stg + lo;
    s->stg_head = hi;
    return cudaSuccess;
}

bool host_pinned(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// memcpy, split over host threads when large (one thread copies a few GB/s;
// a big upload would otherwise keep the host from queueing work).
void host_copy(void* dst, const void* src, size_t bytes) {
    constexpr size_t kPerThread = size_t(4) << 20;
    const unsigned hw = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    const unsigned nt = (unsigned)std::min<size_t>(hw, bytes / kPerThread);
    if (nt <= 1) {
        std::memcpy(dst, src, bytes);
        return;
    }
    std::vector<std::thread> th;
    const size_t per = (bytes / nt + 63) & ~size_t(63);
    for (unsigned t = 0; t < nt; ++t) {
        const size_t lo = std::min(bytes, per * t), hi = std::min(bytes, per * (t + 1));
        if (lo < hi)
            th.emplace_back([=] { std::memcpy(static_cast<char*>(dst) + lo, static_cast<const char*>(src) + lo, hi - lo); });
    }
    for (auto& x : th) x.join();
}

// Copies `bytes` of host data to `dst` in stream order; the caller's buffer
// is free when the call returns and the host never waits for queued work.
// Large copies go through the ring in pieces of kUploadPiece: a ring a few
// pieces long serves a bulk upload of any size (a piece's region is reused
// once its copy has run, which on an idle stream is by the time the host has
// filled the next pieces), instead of pinning a ring as large as the upload.
constexpr size_t kUploadPiece = size_t(16) << 20;
cudaError_t upload_async(nxm_state* s, void* dst, const void* src, size_t bytes) {
    if (bytes == 0) return cudaSuccess;
    if (bytes > kUploadPiece) {
        for (size_t off = 0; off < bytes; off += kUploadPiece) {
            const cudaError_t e = upload_async(s, static_cast<char*>(dst) + off, static_cast<const char*>(src) + off,
                                               std::min(kUploadPiece, bytes - off));
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    char* h = nullptr;
    cudaError_t e = staging_reserve(s, bytes, &h);
    if (e != cudaSuccess) return e;
    host_copy(h, src, bytes);
    e = cudaMemcpyAsync(dst, h, bytes, cudaMemcpyHostToDevice, s->stream);
    if (e != cudaSuccess) return e;
    cudaEvent_t done;
    e = take_event(s, &done);
    if (e != cudaSuccess) return e;
    e = cudaEventRecord(done, s->stream);
    if (e != cudaSuccess) return e;
    s->stg_live.push_back(nxm_state::StagingSpan{(size_t)(h - s->stg), (size_t)(h - s->stg) + bytes, done});
    return cudaSuccess;
}

void invalidate_graph(nxm_state* s) {
    for (int i = 0; i < 2; ++i) {
        if (s->graph[i]) cudaGraphExecDestroy(s->graph[i]);
        s->graph[i] = nullptr;
        s->graph_valid[i] = false;
    }
}

// The reordering G2P wrote the step's output to the *_alt buffers: make them current.
void swap_buffers(nxm_state* s) {
    std::swap(s->kin, s->kin_alt);
    std::swap(s->def, s->def_alt);
    std::swap(s->pstate, s->pstate_alt);
    std::swap(s->pid, s->pid_alt);
    s->parity ^= 1;
}

int grid_for_n(nxm_state* s, uint32_t n) {
    int g = (int)std::min<uint32_t>((n + 255u) / 256u, (uint32_t)s->sm_count * 8u);
    return g < 1 ? 1 : g;
}

// Brings permuted storage back to id order (before edits that address particles by id).
int canonicalize(nxm_state* s) {
    if (!s->permuted) return NXM_OK;
    if (s->n) {
        k_unpermute<<<grid_for_n(s, s->n), 256, 0, s->stream>>>(s->kin, s->def, s->pstate, s->pid, s->n, s->kin_alt,
                                                                 s->def_alt, s->pstate_alt);
        s->launches += 1;
        NXM_TRY(cudaGetLastError());
    }
    std::swap(s->kin, s->kin_alt);
    std::swap(s->def, s->def_alt);
    std::swap(s->pstate, s->pstate_alt);
    std::swap(s->pid, s->pid_alt);
    s->parity ^= 1;
    s->permuted = false;
    NXM_TRY(cudaMemsetAsync(reinterpret_cast<char*>(s->d_counters) + offsetof(Counters, codes_valid), 0, 4,
                            s->stream));
    NXM_TRY(cudaStreamSynchronize(s->stream));
    return NXM_OK;
}

// Arrays carved from one device allocation (each piece 256-byte aligned):
// one cudaMalloc instead of one per array, which is most of the cost of
// creating a state.
struct Slab {
    std::vector<std::pair<void**, size_t>> parts;
    size_t bytes = 0;
    template <class T>
    void add(T** p, size_t count) {
        parts.emplace_back(reinterpret_cast<void**>(p), bytes);
        bytes += (std::max<size_t>(count, 1) * sizeof(T) + 255) & ~size_t(255);
    }
    // Allocates and points every added array into the allocation (or leaves them null).
    cudaError_t alloc(char** base) {
        *base = nullptr;
        if (injected_alloc_failure()) return cudaErrorMemoryAllocation;
        const cudaError_t e = cudaMalloc(reinterpret_cast<void**>(base), bytes);
        if (e != cudaSuccess) {
            *base = nullptr;
            return e;
        }
        for (auto& [ptr, off] : parts) *ptr = *base + off;
        return cudaSuccess;
    }
    void clear() {
        for (auto& [ptr, off] : parts) *ptr = nullptr;
    }
};

void grid_arrays(nxm_state* s, Slab& g) {
    g.add(&s->hkey, s->hash_cap);
    g.add(&s->hval, s->hash_cap);
    g.add(&s->bvid, s->block_cap);
    g.add(&s->first, s->block_cap);
    g.add(&s->nprim, s->block_cap);
    g.add(&s->nwx, s->block_cap);
    g.add(&s->cursors, (size_t)s->block_cap * NUM_BUCKETS);
    g.add(&s->nbh, (size_t)s->block_cap * NUM_NBH);
    g.add(&s->nodes, (size_t)(s->block_cap + 1) * 64);  // + one block of zeros (halos of missing neighbours)
    g.add(&s->scan_tmp, s->block_cap);
    g.add(&s->tile_sums, s->block_cap / kScanTile + 2);
}

int free_grid(nxm_state* s) {
    dfree(s->d_ncdf); dfree(s->d_nodes_inc); dfree(s->d_rp_count); dfree(s->d_rp_first);
    Slab g;
    grid_arrays(s, g);
    g.clear();
    dfree(s->gslab);
    return NXM_OK;
}

// CPIC node fields, sized by the grid capacity.
int alloc_cpic_grid(nxm_state* s) {
    dfree(s->d_ncdf);
    dfree(s->d_nodes_inc);
    dfree(s->d_rp_count);
    dfree(s->d_rp_first);
    NXM_TRY(dalloc(&s->d_ncdf, (size_t)s->block_cap * 64));
    NXM_TRY(dalloc(&s->d_nodes_inc, (size_t)s->block_cap * 64));
    NXM_TRY(dalloc(&s->d_rp_count, s->block_cap));
    NXM_TRY(dalloc(&s->d_rp_first, s->block_cap));
    invalidate_graph(s);
    return NXM_OK;
}

int alloc_grid(nxm_state* s, uint32_t grid_capacity) {
    const uint32_t block_cap = next_pow2(std::max<uint32_t>(grid_capacity, 1));
    if (s->hkey && block_cap == s->block_cap) {  // same capacity: keep the buffers, clear the hash
        NXM_TRY(cudaMemsetAsync(s->hkey, 0xFF, sizeof(uint32_t) * s->hash_cap, s->stream));
        if (s->use_cpic && !s->d_ncdf) {
            int rc = alloc_cpic_grid(s);
            if (rc) return rc;
        }
        invalidate_graph(s);
        s->params_dirty = true;
        return NXM_OK;
    }
    free_grid(s);
    s->block_cap = block_cap;
    s->hash_cap = next_pow2(std::max<uint32_t>(2u * s->block_cap, 1024u));
    Slab g;
    grid_arrays(s, g);
    NXM_TRY(g.alloc(&s->gslab));
    NXM_TRY(cudaMemsetAsync(s->hkey, 0xFF, sizeof(uint32_t) * s->hash_cap, s->stream));
    NXM_TRY(cudaMemsetAsync(s->nodes + (size_t)s->block_cap * 64, 0, 64 * sizeof(float4), s->stream));
    if (s->use_cpic) {
        int rc = alloc_cpic_grid(s);
        if (rc) return rc;
    }
    invalidate_graph(s);
    s->params_dirty = true;
    return NXM_OK;
}

// The particle arrays of a state (owned; freed on destruction unless released).
struct ParticleBuffers {
    char* slab = nullptr;
    PKin *kin = nullptr, *kin_alt = nullptr;
    PDef *def = nullptr, *def_alt = nullptr;
    float4 *pstate = nullptr, *pstate_alt = nullptr;
    uint32_t *pid = nullptr, *pid_alt = nullptr, *phdr = nullptr, *sorted = nullptr, *pscene = nullptr,
             *pscene_alt = nullptr, *tiles = nullptr, *chunk_blk = nullptr;
    uint2* pcode = nullptr;
    float4 *pcdf = nullptr, *pcdf_alt = nullptr;
    cudaError_t alloc(uint32_t cap) {
        Slab a;
        a.add(&kin, cap); a.add(&def, cap); a.add(&pstate, cap);
        a.add(&kin_alt, cap); a.add(&def_alt, cap); a.add(&pstate_alt, cap);
        a.add(&pid, cap); a.add(&pid_alt, cap); a.add(&pcode, cap); a.add(&phdr, cap);
        a.add(&sorted, (size_t)cap * 8);
        a.add(&pscene, cap);
        a.add(&pscene_alt, cap);
        a.add(&pcdf, 3 * (size_t)cap);
        a.add(&pcdf_alt, 3 * (size_t)cap);
        a.add(&tiles, cap / 1024 + 2);
        a.add(&chunk_blk, chunk_cap_for(cap));
        return a.alloc(&slab);
    }
    void release() { *this = ParticleBuffers{}; }
    ~ParticleBuffers() { dfree(slab); }
};

void free_particles(nxm_state* s) {
    dfree(s->pslab);
    s->kin = s->kin_alt = nullptr;
    s->def = s->def_alt = nullptr;
    s->pstate = s->pstate_alt = nullptr;
    s->pid = s->pid_alt = s->phdr = s->sorted = s->d_pscene = s->d_pscene_alt = s->d_tiles = nullptr;
    s->d_chunk_blk = nullptr;
    s->pcode = nullptr;
    s->d_pcdf = s->d_pcdf_alt = nullptr;
}

int invalidate_codes(nxm_state* s);

int reserve_particles(nxm_state* s, uint32_t need) {
    if (need <= s->pcap) return NXM_OK;
    int rc = canonicalize(s);
    if (rc) return rc;
    uint32_t cap = std::max<uint32_t>(need, s->pcap ? s->pcap * 2 : 1024);
    ParticleBuffers t;
    NXM_TRY(t.alloc(cap));
    if (s->n) {
        NXM_TRY(cudaMemcpyAsync(t.kin, s->kin, sizeof(PKin) * s->n, cudaMemcpyDeviceToDevice, s->stream));
        NXM_TRY(cudaMemcpyAsync(t.def, s->def, sizeof(PDef) * s->n, cudaMemcpyDeviceToDevice, s->stream));
        NXM_TRY(cudaMemcpyAsync(t.pstate, s->pstate, sizeof(float4) * s->n, cudaMemcpyDeviceToDevice, s->stream));
        NXM_TRY(cudaMemcpyAsync(t.pscene, s->d_pscene, 4 * (size_t)s->n, cudaMemcpyDeviceToDevice, s->stream));
        NXM_TRY(cudaMemcpyAsync(t.pcdf, s->d_pcdf, 48 * (size_t)s->n, cudaMemcpyDeviceToDevice, s->stream));
    }
    NXM_TRY(cudaStreamSynchronize(s->stream));
    free_particles(s);
    s->pslab = t.slab;
    s->kin = t.kin; s->def = t.def; s->pstate = t.pstate;
    s->kin_alt = t.kin_alt; s->def_alt = t.def_alt; s->pstate_alt = t.pstate_alt;
    s->pid = t.pid; s->pid_alt = t.pid_alt;
    s->pcode = t.pcode; s->phdr = t.phdr; s->sorted = t.sorted;
    s->d_pscene = t.pscene; s->d_pscene_alt = t.pscene_alt; s->d_tiles = t.tiles;
    s->d_pcdf = t.pcdf; s->d_pcdf_alt = t.pcdf_alt;
    s->d_chunk_blk = t.chunk_blk;
    t.release();
    s->sort_pid = nullptr;
    s->pcap = cap;
    invalidate_graph(s);
    s->params_dirty = true;
    // the new arrays hold no cached block keys: the next sort recomputes them
    // from the positions (an upload that fails after this growth leaves the
    // state stepping on these arrays)
    return invalidate_codes(s);
}

// Deduplicates a model's static words; returns the material index.
uint32_t material_of(nxm_state* s, const nxm_particle_model& m) {
    std::vector<uint32_t> key(1 + MODEL_WORDS);
    key[0] = m.tag;
    const int ns = model_state_words(m.tag);
    for (int k = 0; k < MODEL_WORDS; ++k) key[1 + k] = (k < ns) ? 0u : m.data[k];
    auto it = s->material_index.find(key);
    if (it != s->material_index.end()) return it->second;
    Material mat{};
    mat.tag = m.tag;
    mat.has_state = model_has_state(m.tag) ? 1u : 0u;
    for (int k = 0; k < MODEL_WORDS; ++k) mat.w[k] = bits_f(key[1 + k]);
    const uint32_t idx = (uint32_t)s->materials.size();
    s->materials.push_back(mat);
    s->material_index.emplace(std::move(key), idx);
    s->materials_dirty = true;
    return idx;
}

int sync_materials(nxm_state* s) {
    if (!s->materials_dirty) return NXM_OK;
    const uint32_t need = (uint32_t)s->materials.size();
    if (need > s->mat_cap) {
        uint32_t cap = std::max<uint32_t>(need, s->mat_cap ? s->mat_cap * 2 : 16);
        Material* m;
        NXM_TRY(dalloc(&m, cap));
        if (s->d_materials) NXM_TRY(cudaStreamSynchronize(s->stream));  // queued steps may still read it
        dfree(s->d_materials);
        s->d_materials = m;
        s->mat_cap = cap;
        invalidate_graph(s);
    }
    NXM_TRY(upload_async(s, s->d_materials, s->materials.data(), sizeof(Material) * need));
    s->materials_dirty = false;
    return NXM_OK;
}

// The cached block keys (written by the G2P epilogue) no longer match the
// particle positions: the next sort recomputes them from the positions.
int invalidate_codes(nxm_state* s) {
    NXM_TRY(cudaMemsetAsync(reinterpret_cast<char*>(s->d_counters) + offsetof(Counters, codes_valid), 0, 4,
                            s->stream));
    return NXM_OK;
}

int sync_params(nxm_state* s) {
    if (!s->params_dirty) return NXM_OK;
    Params p{};
    p.gravity[0] = s->gravity[0];
    p.gravity[1] = s->gravity[1];
    p.gravity[2] = s->gravity[2];
    p.dt = s->dt;
    p.dx = s->dx;
    p.inv_dx = 1.0f / s->dx;
    p.n = s->n;
    p.ncol = (uint32_t)s->colliders.size();
    p.block_capacity = s->block_cap;
    p.hash_capacity = s->hash_cap;
    p.sorted_capacity = s->pcap * 8u;
    p.use_cpic = s->use_cpic ? 1u : 0u;
    p.scene_blocks = s->scene_blocks;
    p.scene_margin = s->scene_margin;
    for (int k = 0; k < 3; ++k) {
        p.scene_cmin[k] = s->scene_cmin[k];
        p.scene_cells[k] = s->scene_cells[k];
    }
    p.range_min_fill = s->range_min_fill;
    NXM_TRY(upload_async(s, s->d_params, &p, sizeof(Params)));
    s->params_dirty = false;
    return NXM_OK;
}

// Issues the kernels of one step on stream `st`; returns how many.
int enqueue_step(nxm_state* s, cudaStream_t st, cudaEvent_t* ev /* 5 events or null */) {
    DevPtrs P = dev_ptrs(s);
    LaunchCfg c = launch_cfg(s);
    int k = 0;
    const bool has_col = !s->colliders.empty();
    if (ev) cudaEventRecord(ev[0], st);
    // the colliders' centres of mass are refreshed by the sort's first kernel
    // deterministic mode runs the reference's gather-form transfers (with the
    // sort's extras); fast CPIC the scatter P2G with the incompatible split
    const bool exact_path = s->deterministic;
    const bool fast_cpic = !s->deterministic && s->use_cpic;
    const bool rigid = P.nrp > 0;  // CPIC with trimesh colliders
    if (rigid) { exact::launch_rigid_transform(P, c, st); ++k; }  // pipeline.rs:393-405
    fast::launch_sort(P, c, /*with_extras=*/exact_path, /*canonical=*/s->deterministic, st, rigid);
    k += sort_launches(s->deterministic) + (rigid ? fast::kRigidSortLaunches : 0);
    if (s->use_cpic) {  // node and particle distance fields (pipeline.rs:433-460)
        exact::launch_grid_update_cdf(P, c, st);
        if (rigid) { exact::launch_p2g_cdf(P, c, st); ++k; }
        exact::launch_g2p_cdf(P, c, st);
        k += 2;
    }
    if (ev) cudaEventRecord(ev[1], st);
    if (exact_path) exact::launch_p2g_gather(P, c, st);
    else if (fast_cpic) fast::launch_p2g_cpic(P, c, st);
    else fast::launch_p2g(P, c, st);
    k += kP2gLaunches;
    if (ev) cudaEventRecord(ev[2], st);
    if (exact_path) exact::launch_grid_update(P, c, st);
    else if (fast_cpic) fast_cpic::launch_grid_update(P, c, st);
    else fast::launch_grid_update(P, c, st);
    k += kGridLaunches;
    if (ev) cudaEventRecord(ev[3], st);
    k += exact_path   ? exact::launch_g2p_update(P, c, st)
         : fast_cpic ? fast_cpic::launch_g2p_update(P, c, st)
                     : fast::launch_g2p_update(P, c, st);
    if (ev) cudaEventRecord(ev[4], st);
    return k;
}

int ensure_ready(nxm_state* s) {
    int rc = sync_materials(s);
    if (rc) return rc;
    return sync_params(s);
}

// Captures the step for the current buffer parity.
int build_graph(nxm_state* s) {
    const int par = s->parity;
    if (s->graph[par]) cudaGraphExecDestroy(s->graph[par]);
    s->graph[par] = nullptr;
    s->graph_valid[par] = false;
    cudaGraph_t g = nullptr;
    NXM_TRY(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    int k = enqueue_step(s, s->stream, nullptr);
    cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        if (g) cudaGraphDestroy(g);
        return NXM_E_CUDA;
    }
    e = cudaGraphInstantiate(&s->graph[par], g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        s->graph[par] = nullptr;
        return NXM_E_CUDA;
    }
    s->graph_kernels = k;
    s->graph_valid[par] = true;
    return NXM_OK;
}

// Before a reordering step: slot == id unless the storage is already permuted.
int prepare_reorder(nxm_state* s) {
    if (!reorders(s) || s->permuted) return NXM_OK;
    k_iota<<<grid_for_n(s, s->n), 256, 0, s->stream>>>(s->pid, 0u, s->n);
    s->launches += 1;
    NXM_TRY(cudaGetLastError());
    return NXM_OK;
}

// After a step: the sorted ids refer to the slots the step started from.
void finish_step(nxm_state* s) {
    if (reorders(s)) {
        s->sort_pid = s->pid;
        swap_buffers(s);
        s->permuted = true;
    } else {
        s->sort_pid = nullptr;
    }
}

// Fields of particles [first, first + count) (ids), in id order, into `out`.
int pack_read_range(nxm_state* s, const void* records, uint32_t stride_bytes, const int* offsets, int nfields,
                    uint32_t first, uint32_t count, void* out, bool wait = true) {
    if (!out) return NXM_E_INVALID;
    if (first > s->n || count > s->n - first) return NXM_E_INVALID;
    if (count == 0) return NXM_OK;
    const size_t words = (size_t)count * nfields;
    if (words > s->pack_cap) {  // stream-ordered: queued reads of the old scratch finish first
        const size_t cap = std::max(words, s->pack_cap * 2);
        if (s->d_pack) NXM_TRY(cudaFreeAsync(s->d_pack, s->stream));
        s->d_pack = nullptr;
        s->pack_cap = 0;
        NXM_TRY(scratch_alloc(s, &s->d_pack, cap * 4));
        s->pack_cap = cap;
    }
    if (!s->d_offsets) NXM_TRY(dalloc(&s->d_offsets, 32));
    NXM_TRY(upload_async(s, s->d_offsets, offsets, sizeof(int) * nfields));
    const size_t threads = (s->permuted ? (size_t)s->n : (size_t)count) * nfields;
    int grid = (int)std::min<size_t>((threads + 255) / 256, (size_t)s->sm_count * 8);
    if (grid < 1) grid = 1;
    if (s->permuted)
        k_pack_fields_perm<<<grid, 256, 0, s->stream>>>(reinterpret_cast<const uint32_t*>(records), stride_bytes / 4,
                                                          s->n, first, count, s->d_offsets, nfields, s->pid,
                                                          s->d_pack);
    else
        k_pack_fields<<<grid, 256, 0, s->stream>>>(reinterpret_cast<const uint32_t*>(records), stride_bytes / 4, first,
                                                     count, s->d_offsets, nfields, s->d_pack);
    s->launches += 1;
    NXM_TRY(cudaGetLastError());
    NXM_TRY(cudaMemcpyAsync(out, s->d_pack, words * 4, cudaMemcpyDeviceToHost, s->stream));
    if (wait) NXM_TRY(cudaStreamSynchronize(s->stream));
    return NXM_OK;
}

int pack_read(nxm_state* s, const void* records, uint32_t stride_bytes, const int* offsets, int nfields, void* out) {
    if (!out) return NXM_E_INVALID;
    return pack_read_range(s, records, stride_bytes, offsets, nfields, 0, s->n, out);
}

// Removes the particles whose ids fall in `ranges` (sorted, disjoint), keeping
// the others in their relative order (ids shift down), on canonical or
// block-ordered storage alike: one compaction pass over the storage slots into
// the other buffers, which then become current.  Host mirrors follow.
int remove_id_ranges(nxm_state* s, std::vector<uint2> ranges) {
    std::sort(ranges.begin(), ranges.end(), [](uint2 a, uint2 b) { return a.x < b.x; });
    std::vector<uint2> rr;
    for (uint2 r : ranges) {
        r.y = std::min(r.y, s->n);
        if (r.x >= r.y) continue;
        if (!rr.empty() && r.x < rr.back().y) return NXM_E_INVALID;  // overlapping ranges
        rr.push_back(r);
    }
    if (rr.empty()) return NXM_OK;
    std::vector<uint32_t> cum(rr.size());
    uint32_t removed = 0;
    for (size_t i = 0; i < rr.size(); ++i) {
        cum[i] = removed;
        removed += rr[i].y - rr[i].x;
    }
    const uint32_t n0 = s->n, ntiles = (n0 + 1023u) / 1024u;
    // stream-ordered scratch and staged uploads: the removal queues behind the
    // steps in flight without waiting for them
    char* scratch = nullptr;
    cudaError_t e = scratch_alloc(s, &scratch, 16 * rr.size() + 16);
    uint2* d_r = reinterpret_cast<uint2*>(scratch);
    uint32_t* d_cum = reinterpret_cast<uint32_t*>(scratch + 8 * rr.size());
    if (e == cudaSuccess) e = upload_async(s, d_r, rr.data(), sizeof(uint2) * rr.size());
    if (e == cudaSuccess) e = upload_async(s, d_cum, cum.data(), 4 * cum.size());
    const uint32_t* pid = s->permuted ? s->pid : nullptr;
    const uint32_t nr = (uint32_t)rr.size();
    if (e == cudaSuccess) {
        k_rm_count<<<ntiles, 256, 0, s->stream>>>(n0, pid, d_r, nr, s->d_tiles);
        k_rm_scan<<<1, 1024, 0, s->stream>>>(s->d_tiles, ntiles);
        k_rm_move<<<ntiles, 256, 0, s->stream>>>(n0, s->kin, s->def, s->pstate, pid, d_r, d_cum, nr, s->d_tiles,
                                                 s->kin_alt, s->def_alt, s->pstate_alt, s->pid_alt);
        s->launches += 3;
        if (s->scene_blocks) {  // the per-id scene index follows the ids
            k_rm_ids<uint32_t, 1><<<grid_for_n(s, n0), 256, 0, s->stream>>>(n0, s->d_pscene, d_r, d_cum, nr,
                                                                             s->d_pscene_alt);
            s->launches += 1;
        }
        k_rm_ids<float4, 3><<<grid_for_n(s, n0), 256, 0, s->stream>>>(n0, s->d_pcdf, d_r, d_cum, nr, s->d_pcdf_alt);
        s->launches += 1;
        e = cudaGetLastError();
    }
    if (scratch) cudaFreeAsync(scratch, s->stream);
    NXM_TRY(e);
    swap_buffers(s);  // the compacted records (and, when permuted, their ids) are current
    if (s->scene_blocks) std::swap(s->d_pscene, s->d_pscene_alt);
    std::swap(s->d_pcdf, s->d_pcdf_alt);
    if (s->chunks_used) {
        for (size_t i = rr.size(); i-- > 0;)
            s->slot2chunk.erase(s->slot2chunk.begin() + rr[i].x, s->slot2chunk.begin() + rr[i].y);
        for (auto& c : s->chunks) c.second = 0;  // recount chunk sizes
        for (uint32_t o : s->slot2chunk)
            if (o != NONE) {
                auto it = s->chunks.find(o);
                if (it != s->chunks.end()) ++it->second;
            }
    }
    s->n = n0 - removed;
    s->sort_pid = nullptr;
    s->params_dirty = true;
    return invalidate_codes(s);
}

// Material runs of an upload: consecutive particles with byte-identical models
// share one material and one initial model state (a new run starts wherever
// the model differs from the previous particle's).  The comparison runs in
// parallel over slices of the particles; the lookups, one per run, serially.
struct MaterialRuns {
    std::vector<uint32_t> start, mid;
    std::vector<float4> state;
};

static int material_runs(nxm_state* s, const nxm_particle_model* models, uint32_t count, MaterialRuns& r) {
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const uint32_t nt = count < (1u << 16) ? 1u : hw;
    std::vector<std::vector<uint32_t>> starts(nt);
    auto scan = [&](uint32_t t) {
        const uint32_t lo = (uint32_t)((uint64_t)count * t / nt), hi = (uint32_t)((uint64_t)count * (t + 1) / nt);
        for (uint32_t i = lo; i < hi; ++i)
            if (i == 0 || std::memcmp(&models[i], &models[i - 1], sizeof(nxm_particle_model)) != 0)
                starts[t].push_back(i);
    };
    if (nt == 1) {
        scan(0);
    } else {
        std::vector<std::thread> th;
        for (uint32_t t = 0; t < nt; ++t) th.emplace_back(scan, t);
        for (auto& x : th) x.join();
    }
    for (const auto& v : starts) r.start.insert(r.start.end(), v.begin(), v.end());
    r.mid.resize(r.start.size());
    r.state.resize(r.start.size());
    for (size_t k = 0; k < r.start.size(); ++k) {
        const nxm_particle_model& m = models[r.start[k]];
        r.mid[k] = material_of(s, m);
        float st[4] = {0, 0, 0, 0};
        for (int w = 0; w < model_state_words(m.tag); ++w) st[w] = bits_f(m.data[w]);
        r.state[k] = make_float4(st[0], st[1], st[2], st[3]);
    }
    return NXM_OK;
}

// Device-side record packing of an upload: the SoA fields (null = the
// ParticleDynamics::new default) of particles [base, base + count) of the
// upload, written as PKin / PDef / model state / CPIC + properties records.
struct UploadSrc {
    const float *pos, *vel, *F, *A, *vgd, *v0, *rad, *mass, *damp, *phase, *bf;
    const uint32_t *gid, *en, *fx;
    const uint32_t* run_start;
    const uint32_t* run_mid;
    const float4* run_state;
    uint32_t nruns;
};

__global__ void k_pack_particles(UploadSrc u, uint32_t base, uint32_t count, PKin* __restrict__ kin,
                                 PDef* __restrict__ def, float4* __restrict__ pstate, float4* __restrict__ pcdf) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        // the material run holding particle base + i
        uint32_t lo = 0, hi = u.nruns;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (u.run_start[mid] <= base + i) lo = mid; else hi = mid;
        }
        const float* x = u.pos + 3 * (size_t)i;
        const float* v = u.vel ? u.vel + 3 * (size_t)i : nullptr;
        const float* a = u.A ? u.A + 9 * (size_t)i : nullptr;
        const float* F = u.F ? u.F + 9 * (size_t)i : nullptr;
        uint32_t flags = 0;
        if (!u.en || u.en[i]) flags |= PFLAG_ENABLED;
        if (u.fx && u.fx[i]) flags |= PFLAG_FIXED;
        float4* k = reinterpret_cast<float4*>(&kin[i]);
        k[0] = make_float4(x[0], x[1], x[2], u.mass[i]);
        k[1] = make_float4(v ? v[0] : 0.f, v ? v[1] : 0.f, v ? v[2] : 0.f, __uint_as_float(flags));
        k[2] = make_float4(a ? a[0] : 0.f, a ? a[1] : 0.f, a ? a[2] : 0.f, u.vgd ? u.vgd[i] : 0.f);
        k[3] = make_float4(a ? a[3] : 0.f, a ? a[4] : 0.f, a ? a[5] : 0.f, 0.f);
        k[4] = make_float4(a ? a[6] : 0.f, a ? a[7] : 0.f, a ? a[8] : 0.f, 0.f);
        float4* d = reinterpret_cast<float4*>(&def[i]);
        d[0] = make_float4(F ? F[0] : 1.f, F ? F[1] : 0.f, F ? F[2] : 0.f, u.v0[i]);
        d[1] = make_float4(F ? F[3] : 0.f, F ? F[4] : 1.f, F ? F[5] : 0.f, u.damp ? u.damp[i] : 0.f);
        d[2] = make_float4(F ? F[6] : 0.f, F ? F[7] : 0.f, F ? F[8] : 1.f, __uint_as_float(u.run_mid[lo]));
        pstate[i] = u.run_state[lo];
        // CPIC fields start empty; then the properties: defaults of
        // ParticleDynamics::new (solver/particle.rs:100-122), the radius, when
        // not given, from init_volume = (2 r)^3
        pcdf[3 * (size_t)i] = make_float4(0.f, 0.f, 0.f, 0.f);
        pcdf[3 * (size_t)i + 1] = make_float4(0.f, 0.f, 0.f, 0.f);
        pcdf[3 * (size_t)i + 2] = make_float4(u.bf ? u.bf[i] : 1.0f, u.rad ? u.rad[i] : 0.5f * cbrtf(u.v0[i]),
                                              u.phase ? u.phase[i] : 1.0f, __uint_as_float(u.gid ? u.gid[i] : 0u));
    }
}

// Appends `count` particles: the caller's SoA arrays are copied as they are
// into a stream-ordered scratch, chunk by chunk, and packed into the particle
// records on the device; only the material runs are resolved on the host.
// Arrays in pinned memory are copied directly (the call then waits for the
// copies before returning, as the caller owns them); pageable ones go through
// the staging ring, so the upload is queued behind the running steps without
// the host waiting for them.
int upload_particles(nxm_state* s, const nxm_particles_soa* p, uint32_t count) {
    if (count == 0) return NXM_OK;
    if (!p || !p->position || !p->model) return NXM_E_INVALID;
    if ((!p->init_volume || !p->mass)) return NXM_E_INVALID;
    uint64_t need = (uint64_t)s->n + count;
    if (need > 0x7FFFFFFFull / 8) return NXM_E_INVALID;
    int rc = reserve_particles(s, (uint32_t)need);
    if (rc) return rc;

    // scratch for one chunk of the fields that are given
    const uint32_t chunk = std::min<uint32_t>(count, 1u << 20);
    struct Field {
        const void* src;
        size_t elem;  // bytes per particle
    };
    const Field fields[14] = {{p->position, 12}, {p->velocity, 12}, {p->def_grad, 36},   {p->affine, 36},
                              {p->vel_grad_det, 4}, {p->init_volume, 4}, {p->init_radius, 4}, {p->mass, 4},
                              {p->damping, 4},  {p->phase, 4},     {p->boundary_friction, 4}, {p->group_id, 4},
                              {p->enabled, 4},  {p->fixed, 4}};
    size_t per_particle = 0;
    for (const Field& f : fields)
        if (f.src) per_particle += f.elem;
    bool pinned[14] = {};
    bool direct = false;  // some copy reads the caller's pinned memory
    for (int f = 0; f < 14; ++f)
        if (fields[f].src) direct |= (pinned[f] = host_pinned(fields[f].src));
    char* scratch = nullptr;
    NXM_TRY(scratch_alloc(s, &scratch, std::max<size_t>(per_particle, 4) * chunk));
    const void* dst[14] = {};
    auto copy_chunk = [&](uint32_t c0, uint32_t cn) {
        char* at = scratch;
        cudaError_t e = cudaSuccess;
        for (int f = 0; f < 14 && e == cudaSuccess; ++f) {
            dst[f] = nullptr;
            if (!fields[f].src) continue;
            dst[f] = at;
            const char* from = static_cast<const char*>(fields[f].src) + fields[f].elem * c0;
            e = pinned[f] ? cudaMemcpyAsync(at, from, fields[f].elem * cn, cudaMemcpyHostToDevice, s->stream)
                          : upload_async(s, at, from, fields[f].elem * cn);
            at += fields[f].elem * chunk;
        }
        return e;
    };
    // The first chunk's copies are queued before the host looks for the
    // material runs, so the scan over the model words overlaps the transfer.
    cudaError_t err = copy_chunk(0, std::min(chunk, count));
    MaterialRuns runs;
    if (err == cudaSuccess) rc = material_runs(s, p->model, count, runs);
    else rc = NXM_E_CUDA;
    if (!rc) rc = sync_materials(s);
    char* run_scratch = nullptr;
    UploadSrc u{};
    if (!rc) {
        const uint32_t nruns = (uint32_t)runs.start.size();
        const size_t mid_at = (size_t)nruns * 4, state_at = ((size_t)nruns * 8 + 15) / 16 * 16;
        cudaError_t e = scratch_alloc(s, &run_scratch, state_at + (size_t)nruns * 16);
        if (e == cudaSuccess) e = upload_async(s, run_scratch, runs.start.data(), 4 * (size_t)nruns);
        if (e == cudaSuccess) e = upload_async(s, run_scratch + mid_at, runs.mid.data(), 4 * (size_t)nruns);
        if (e == cudaSuccess) e = upload_async(s, run_scratch + state_at, runs.state.data(), 16 * (size_t)nruns);
        if (e != cudaSuccess) rc = NXM_E_CUDA;
        u.nruns = nruns;
        u.run_start = reinterpret_cast<const uint32_t*>(run_scratch);
        u.run_mid = reinterpret_cast<const uint32_t*>(run_scratch + mid_at);
        u.run_state = reinterpret_cast<const float4*>(run_scratch + state_at);
    }
    if (rc) {
        cudaFreeAsync(scratch, s->stream);
        if (run_scratch) cudaFreeAsync(run_scratch, s->stream);
        if (direct) (void)cudaStreamSynchronize(s->stream);  // no copy reads the caller's memory after return
        (void)cudaGetLastError();
        return rc;
    }
    if (s->chunks_used) s->slot2chunk.insert(s->slot2chunk.end(), count, NONE);
    for (uint32_t c0 = 0; c0 < count && err == cudaSuccess; c0 += chunk) {
        const uint32_t cn = std::min(chunk, count - c0);
        if (c0 > 0) err = copy_chunk(c0, cn);  // queued after the previous chunk's packing
        if (err != cudaSuccess) break;
        u.pos = static_cast<const float*>(dst[0]);
        u.vel = static_cast<const float*>(dst[1]);
        u.F = static_cast<const float*>(dst[2]);
        u.A = static_cast<const float*>(dst[3]);
        u.vgd = static_cast<const float*>(dst[4]);
        u.v0 = static_cast<const float*>(dst[5]);
        u.rad = static_cast<const float*>(dst[6]);
        u.mass = static_cast<const float*>(dst[7]);
        u.damp = static_cast<const float*>(dst[8]);
        u.phase = static_cast<const float*>(dst[9]);
        u.bf = static_cast<const float*>(dst[10]);
        u.gid = static_cast<const uint32_t*>(dst[11]);
        u.en = static_cast<const uint32_t*>(dst[12]);
        u.fx = static_cast<const uint32_t*>(dst[13]);
        const size_t at0 = (size_t)s->n + c0;
        k_pack_particles<<<grid_for_n(s, cn), 256, 0, s->stream>>>(u, c0, cn, s->kin + at0, s->def + at0,
                                                                   s->pstate + at0, s->d_pcdf + 3 * at0);
        s->launches += 1;
        err = cudaGetLastError();
    }
    cudaFreeAsync(scratch, s->stream);
    cudaFreeAsync(run_scratch, s->stream);
    if (err != cudaSuccess) {
        if (direct) (void)cudaStreamSynchronize(s->stream);
        return NXM_E_CUDA;
    }
    if (s->permuted) {  // appended particles sit at slots == their ids
        k_iota<<<grid_for_n(s, count), 256, 0, s->stream>>>(s->pid + s->n, s->n, count);
        s->launches += 1;
        NXM_TRY(cudaGetLastError());
    }
    if (direct) NXM_TRY(cudaStreamSynchronize(s->stream));
    s->n += count;
    s->params_dirty = true;
    return invalidate_codes(s);
}

// ---- trimesh colliders (host side) ------------------------------------------

using VKey = std::array<uint32_t, 3>;  // vertex position, bit pattern

VKey vkey(const float* v) { return VKey{f_bits(v[0]), f_bits(v[1]), f_bits(v[2])}; }

// Triangle records with pseudo-normals for the triangles [first, first + count)
// of `tri` (9 floats each), treated as one mesh: the pseudo-normal of a vertex
// sums, over the mesh's non-degenerate triangles with a vertex at that exact
// position, the unit face normal times the corner angle; that of an edge sums
// the unit normals of the triangles sharing it (either orientation); that of
// the face is ab x ac.  These are the pseudo-normals the reference uploads
// per vertex and per triangle edge (rbd shapes/trimesh.rs:111-150).
void trimesh_records(const float* tri, uint32_t first, uint32_t count, std::vector<DevTri>& out) {
    std::map<VKey, std::array<double, 3>> vpn;
    std::map<std::pair<VKey, VKey>, std::array<double, 3>> epn;
    auto sub = [](const float* a, const float* b, double* r) {
        for (int k = 0; k < 3; ++k) r[k] = (double)a[k] - (double)b[k];
    };
    auto ekey = [](const VKey& a, const VKey& b) { return a < b ? std::make_pair(a, b) : std::make_pair(b, a); };
    for (uint32_t t = first; t < first + count; ++t) {
        const float* q[3] = {tri + 9 * (size_t)t, tri + 9 * (size_t)t + 3, tri + 9 * (size_t)t + 6};
        double u[3], w[3];
        sub(q[1], q[0], u);
        sub(q[2], q[0], w);
        double fn[3] = {u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]};
        const double fl = std::sqrt(fn[0] * fn[0] + fn[1] * fn[1] + fn[2] * fn[2]);
        if (fl == 0.0) continue;
        for (double& x : fn) x /= fl;
        for (int k = 0; k < 3; ++k) {
            double e0[3], e1[3];
            sub(q[(k + 1) % 3], q[k], e0);
            sub(q[(k + 2) % 3], q[k], e1);
            const double l0 = std::sqrt(e0[0] * e0[0] + e0[1] * e0[1] + e0[2] * e0[2]);
            const double l1 = std::sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
            double c = (e0[0] * e1[0] + e0[1] * e1[1] + e0[2] * e1[2]) / (l0 * l1);
            c = std::min(1.0, std::max(-1.0, c));
            const double ang = std::acos(c);
            auto& a = vpn[vkey(q[k])];
            for (int d = 0; d < 3; ++d) a[d] += fn[d] * ang;
            auto& e = epn[ekey(vkey(q[k]), vkey(q[(k + 1) % 3]))];
            for (int d = 0; d < 3; ++d) e[d] += fn[d];
        }
    }
    for (uint32_t t = first; t < first + count; ++t) {
        const float* q[3] = {tri + 9 * (size_t)t, tri + 9 * (size_t)t + 3, tri + 9 * (size_t)t + 6};
        DevTri r{};
        for (int k = 0; k < 3; ++k)
            for (int d = 0; d < 3; ++d) r.v[k][d] = q[k][d];
        for (int k = 0; k < 3; ++k) {
            auto it = vpn.find(vkey(q[k]));
            auto ie = epn.find(ekey(vkey(q[k]), vkey(q[(k + 1) % 3])));
            for (int d = 0; d < 3; ++d) {
                r.pn[k][d] = it == vpn.end() ? 0.f : (float)it->second[d];
                r.pn[3 + k][d] = ie == epn.end() ? 0.f : (float)ie->second[d];
            }
        }
        double u[3], w[3];
        sub(q[1], q[0], u);
        sub(q[2], q[0], w);
        r.pn[6][0] = (float)(u[1] * w[2] - u[2] * w[1]);
        r.pn[6][1] = (float)(u[2] * w[0] - u[0] * w[2]);
        r.pn[6][2] = (float)(u[0] * w[1] - u[1] * w[0]);
        out.push_back(r);
    }
}

// Skip-link BVH over the records [base, base + count) of `tris`: median split
// of the triangle centroids along the longest axis of their bounds, one
// triangle per leaf, nodes in depth-first order starting at node index `node0`.
struct BvhItem {
    float mn[3], mx[3], c[3];
    uint32_t tri;
};
uint32_t bvh_build(std::vector<BvhItem>& items, size_t lo, size_t hi, uint32_t node0, std::vector<DevBvhNode>& nodes) {
    const uint32_t id = (uint32_t)nodes.size();
    nodes.push_back(DevBvhNode{});
    DevBvhNode n{};
    float cmn[3], cmx[3];
    for (int d = 0; d < 3; ++d) {
        n.mn[d] = cmn[d] = 3.0e38f;
        n.mx[d] = cmx[d] = -3.0e38f;
    }
    for (size_t i = lo; i < hi; ++i)
        for (int d = 0; d < 3; ++d) {
            n.mn[d] = std::min(n.mn[d], items[i].mn[d]);
            n.mx[d] = std::max(n.mx[d], items[i].mx[d]);
            cmn[d] = std::min(cmn[d], items[i].c[d]);
            cmx[d] = std::max(cmx[d], items[i].c[d]);
        }
    if (hi - lo == 1) {
        n.entry = kBvhLeaf | items[lo].tri;
    } else {
        int axis = 0;
        for (int d = 1; d < 3; ++d)
            if (cmx[d] - cmn[d] > cmx[axis] - cmn[axis]) axis = d;
        const size_t mid = lo + (hi - lo) / 2;
        std::nth_element(items.begin() + lo, items.begin() + mid, items.begin() + hi,
                         [axis](const BvhItem& a, const BvhItem& b) { return a.c[axis] < b.c[axis]; });
        n.entry = node0 + id + 1;
        bvh_build(items, lo, mid, node0, nodes);
        bvh_build(items, mid, hi, node0, nodes);
    }
    n.exit = node0 + (uint32_t)nodes.size();
    nodes[id] = n;
    return id;
}

void trimesh_bvh(const std::vector<DevTri>& tris, uint32_t base, uint32_t count, uint32_t node0,
                 std::vector<DevBvhNode>& nodes) {
    std::vector<BvhItem> items(count);
    for (uint32_t i = 0; i < count; ++i) {
        const DevTri& t = tris[base + i];
        BvhItem& it = items[i];
        for (int d = 0; d < 3; ++d) {
            it.mn[d] = std::min(t.v[0][d], std::min(t.v[1][d], t.v[2][d]));
            it.mx[d] = std::max(t.v[0][d], std::max(t.v[1][d], t.v[2][d]));
            it.c[d] = (t.v[0][d] + t.v[1][d] + t.v[2][d]) / 3.0f;
        }
        it.tri = base + i;
    }
    std::vector<DevBvhNode> local;
    local.reserve(2 * (size_t)count);
    bvh_build(items, 0, count, node0, local);
    nodes.insert(nodes.end(), local.begin(), local.end());
}

// ---- CPIC rigid particles (host side) ------------------------------------------
//
// src_mpm/sampling/sample_trimesh.rs:66-231 sample_mesh, in f32 operation by
// operation (this file is built with -ffp-contract=off): per triangle, rows
// perpendicular to its longest edge every step / sqrt(2) with points every
// step / sqrt(2) along each row (none on the edges), then each edge not seen
// before (vertices identified by their position bits) sampled every
// step / sqrt(2) from its first vertex (excluded).  The sampling step is the
// cell width (solver/particle.rs:296-349).

constexpr float kSampleEps = 1.0e-5f;

struct F3 {
    float x, y, z;
};
static inline F3 f3sub(F3 a, F3 b) { return F3{a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline F3 f3add(F3 a, F3 b) { return F3{a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline F3 f3mul(F3 a, float s) { return F3{a.x * s, a.y * s, a.z * s}; }
static inline F3 f3div(F3 a, float s) { return F3{a.x / s, a.y / s, a.z / s}; }
static inline float f3dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float f3len(F3 a) { return std::sqrt(f3dot(a, a)); }
// Rust `f32 as u32`: saturating, NaN -> 0.
static inline uint32_t count_of(float f) {
    return !(f > 0.0f) ? 0u : (f >= 4294967295.0f ? 0xFFFFFFFFu : (uint32_t)f);
}

struct RigidSample {
    F3 p;
    uint32_t tri;  // index into the state's triangle records
};

void sample_edge(F3 a, F3 b, float step, uint32_t tri, std::vector<RigidSample>& out) {
    const F3 ab = f3sub(b, a);
    const float len = f3len(ab);
    if (!(len > kSampleEps)) return;
    const F3 dir = f3div(ab, len);
    const float spacing = step / std::sqrt(2.0f);
    const uint32_t n = count_of(std::ceil(len / spacing));
    for (uint32_t i = 1; i < n; ++i) out.push_back(RigidSample{f3add(a, f3mul(dir, spacing * (float)i)), tri});
}

void sample_triangle(F3 a, F3 b, F3 c, float step, uint32_t tri, std::vector<RigidSample>& out) {
    const float d_ab = f3len(f3sub(b, a)), d_bc = f3len(f3sub(c, b)), d_ca = f3len(f3sub(a, c));
    const float mx = std::fmax(std::fmax(d_ab, d_bc), d_ca);
    if (mx == d_bc) {
        const F3 t = a; a = b; b = c; c = t;
    } else if (mx == d_ca) {
        const F3 t = a; a = c; c = b; b = t;
    }
    const F3 ac = f3sub(c, a), base = f3sub(b, a);
    const float base_length = f3len(base);
    const F3 base_dir = f3div(base, base_length);
    const float spacing = step / std::sqrt(2.0f);
    const float base_steps = std::ceil(base_length / spacing);
    const F3 base_step = f3mul(base_dir, spacing);
    const float ac_off = f3dot(ac, base_dir);
    const float bc_off = base_length - ac_off;
    if (ac_off < kSampleEps || bc_off < kSampleEps || base_length < kSampleEps) return;
    const F3 height = f3sub(ac, f3mul(base_dir, ac_off));
    const float height_length = f3len(height);
    const F3 height_dir = f3div(height, height_length);
    const float tan_a = height_length / ac_off, tan_b = height_length / bc_off;
    const uint32_t nb = count_of(base_steps);
    for (uint32_t i = 1; i < nb; ++i) {
        const F3 bp = f3add(a, f3mul(base_step, (float)i));
        const float h_ac = tan_a * f3len(f3sub(a, bp));
        const float h_bc = tan_b * f3len(f3sub(b, bp));
        const float hl = std::fmin(h_ac, h_bc);
        const uint32_t nh = count_of(std::ceil(hl / spacing));
        const F3 hstep = f3mul(height_dir, spacing);
        for (uint32_t j = 1; j < nh; ++j) {
            const F3 pp = f3add(bp, f3mul(hstep, (float)j));
            if (!std::isfinite(pp.x) || !std::isfinite(pp.y) || !std::isfinite(pp.z)) continue;
            out.push_back(RigidSample{pp, tri});
        }
    }
}

// Samples of the triangle records [base, base + count) (one mesh).
void sample_mesh(const std::vector<DevTri>& tris, uint32_t base, uint32_t count, float step,
                 std::vector<RigidSample>& out) {
    std::map<VKey, uint32_t> vid;
    std::set<std::pair<uint32_t, uint32_t>> seen;
    auto id_of = [&vid](const float* v) {
        auto it = vid.emplace(vkey(v), (uint32_t)vid.size());
        return it.first->second;
    };
    auto first_visit = [&seen](uint32_t a, uint32_t b) {
        return seen.insert(a < b ? std::make_pair(a, b) : std::make_pair(b, a)).second;
    };
    for (uint32_t t = base; t < base + count; ++t) {
        const DevTri& r = tris[t];
        const F3 q[3] = {F3{r.v[0][0], r.v[0][1], r.v[0][2]}, F3{r.v[1][0], r.v[1][1], r.v[1][2]},
                         F3{r.v[2][0], r.v[2][1], r.v[2][2]}};
        const uint32_t i0 = id_of(r.v[0]), i1 = id_of(r.v[1]), i2 = id_of(r.v[2]);
        sample_triangle(q[0], q[1], q[2], step, t, out);
        if (first_visit(i0, i1)) sample_edge(q[0], q[1], step, t, out);
        if (first_visit(i1, i2)) sample_edge(q[1], q[2], step, t, out);
        if (first_visit(i2, i0)) sample_edge(q[2], q[0], step, t, out);
    }
}

// Device form of one nxm_collider (triangle indices shifted by `tri_offset`).
int collider_from_abi(const nxm_collider& c, const float* tri, uint32_t ntri, uint32_t tri_offset, DevCollider& d) {
    std::memset(&d, 0, sizeof(d));
    d.scene = NONE;
    std::memcpy(d.a, c.shape_a, 16);
    std::memcpy(d.b, c.shape_b, 16);
    std::memcpy(d.c, c.shape_c, 16);
    std::memcpy(d.rot, c.rotation, 16);
    std::memcpy(d.tra, c.translation, 12);
    std::memcpy(d.linvel, c.linvel, 12);
    std::memcpy(d.angvel, c.angvel, 12);
    std::memcpy(d.local_com, c.local_com, 12);
    d.type = f_bits(c.shape_a[3]);
    d.bc_type = c.bc_type;
    d.bc_friction = c.bc_friction;
    d.tri_first = c.tri_first + tri_offset;
    d.tri_count = c.tri_count;
    if (d.type != SHAPE_BALL && d.type != SHAPE_CUBOID && d.type != SHAPE_CAPSULE && d.type != SHAPE_TRIMESH)
        return NXM_E_UNSUPPORTED;
    if (d.type == SHAPE_TRIMESH && (!tri || c.tri_count == 0 || c.tri_first > ntri || c.tri_count > ntri - c.tri_first))
        return NXM_E_INVALID;
    return NXM_OK;
}

// Uploads the collider table (every trimesh gets its own triangle records and
// BVH, built from `tri`), growing the device table when needed.
int rebuild_rigid_particles(nxm_state* s);

int install_colliders(nxm_state* s, std::vector<DevCollider> dc, const float* tri) {
    std::vector<DevTri> tris;
    std::vector<DevBvhNode> bvh;
    std::vector<uint32_t> tri_base(dc.size(), 0u);
    for (size_t i = 0; i < dc.size(); ++i) {
        DevCollider& d = dc[i];
        if (d.type != SHAPE_TRIMESH) continue;
        const uint32_t base = (uint32_t)tris.size();
        tri_base[i] = base;
        trimesh_records(tri, d.tri_first, d.tri_count, tris);
        d.bvh_first = (uint32_t)bvh.size();
        trimesh_bvh(tris, base, d.tri_count, d.bvh_first, bvh);
        d.bvh_count = (uint32_t)bvh.size() - d.bvh_first;
    }
    // buffers the queued steps read are replaced only after they ran; a table
    // that fits is rewritten in stream order, without waiting
    const bool had_mesh = s->d_tris != nullptr;
    const bool replace = dc.size() > s->col_cap || had_mesh || !tris.empty();
    if (replace) NXM_TRY(cudaStreamSynchronize(s->stream));
    bool realloc_graph = false;
    if (dc.size() > s->col_cap) {
        const uint32_t cap = std::max<uint32_t>((uint32_t)dc.size(), 2 * s->col_cap);
        DevCollider* d = nullptr;
        NXM_TRY(dalloc(&d, cap));
        dfree(s->d_colliders);
        s->d_colliders = d;
        s->col_cap = cap;
        realloc_graph = true;
    }
    if (!dc.empty()) NXM_TRY(upload_async(s, s->d_colliders, dc.data(), sizeof(DevCollider) * dc.size()));
    if (replace) {
        dfree(s->d_tris);
        dfree(s->d_bvh);
        if (!tris.empty()) {
            NXM_TRY(dalloc(&s->d_tris, tris.size()));
            NXM_TRY(dalloc(&s->d_bvh, bvh.size()));
            NXM_TRY(upload_async(s, s->d_tris, tris.data(), sizeof(DevTri) * tris.size()));
            NXM_TRY(upload_async(s, s->d_bvh, bvh.data(), sizeof(DevBvhNode) * bvh.size()));
        }
    }
    const bool had = !s->colliders.empty();
    s->colliders = dc;
    s->tris_host = std::move(tris);
    s->tri_base = std::move(tri_base);
    if (realloc_graph || had != !s->colliders.empty() || had_mesh || !s->tris_host.empty()) invalidate_graph(s);
    s->params_dirty = true;
    return rebuild_rigid_particles(s);
}

// (Re)samples the CPIC rigid particles of the trimesh colliders (none
// without CPIC), as the reference does when the coupling is set
// (src_mpm/pipeline.rs:211-245).
int rebuild_rigid_particles(nxm_state* s) {
    if (!s->use_cpic && s->nrp == 0) return NXM_OK;  // nothing sampled, nothing to free
    NXM_TRY(cudaStreamSynchronize(s->stream));
    dfree(s->d_rp_local); dfree(s->d_rp_world); dfree(s->d_rp_need); dfree(s->d_rp_sorted);
    const bool had = s->nrp != 0;
    s->nrp = 0;
    s->rp_host.clear();
    if (s->use_cpic) {
        if (s->tris_host.size() > kRigidTriMask) return NXM_E_INVALID;
        std::vector<RigidSample> smp;
        for (size_t i = 0; i < s->colliders.size(); ++i) {
            const DevCollider& d = s->colliders[i];
            if (d.type != SHAPE_TRIMESH) continue;
            const size_t before = smp.size();
            sample_mesh(s->tris_host, s->tri_base[i], d.tri_count, s->dx, smp);
            for (size_t k = before; k < smp.size(); ++k) {
                const RigidSample& r = smp[k];
                s->rp_host.push_back(make_float4(r.p.x, r.p.y, r.p.z, bits_f(r.tri | ((uint32_t)i << kRigidTriBits))));
            }
        }
        if (s->rp_host.size() > (size_t)UINT32_MAX / 8) return NXM_E_INVALID;
        s->nrp = (uint32_t)s->rp_host.size();
    }
    if (s->nrp) {
        NXM_TRY(dalloc(&s->d_rp_local, s->nrp));
        NXM_TRY(dalloc(&s->d_rp_world, s->nrp));
        NXM_TRY(dalloc(&s->d_rp_need, s->nrp));
        NXM_TRY(dalloc(&s->d_rp_sorted, 8 * (size_t)s->nrp));
        NXM_TRY(cudaMemcpyAsync(s->d_rp_local, s->rp_host.data(), sizeof(float4) * s->nrp, cudaMemcpyHostToDevice,
                                s->stream));
        // world = local until the first step (solver/particle.rs:272-276)
        NXM_TRY(cudaMemcpyAsync(s->d_rp_world, s->d_rp_local, sizeof(float4) * s->nrp, cudaMemcpyDeviceToDevice,
                                s->stream));
        NXM_TRY(cudaStreamSynchronize(s->stream));
    }
    if (had || s->nrp) invalidate_graph(s);
    return NXM_OK;
}

bool device_ok(int* dev, int* sms) {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        (void)cudaGetLastError();
        return false;
    }
    int d = 0, major = 0, count_sm = 0;
    if (cudaGetDevice(&d) != cudaSuccess) return false;
    // two attribute queries (a full property query costs milliseconds)
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, d) != cudaSuccess) return false;
    if (cudaDeviceGetAttribute(&count_sm, cudaDevAttrMultiProcessorCount, d) != cudaSuccess) return false;
    if (major != 10) return false;  // kernels are built for sm_100a only
    *dev = d;
    *sms = count_sm;
    return true;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================

extern "C" {

const char* nxm_error_string(int code) {
    switch (code) {
    case NXM_OK: return "ok";
    case NXM_E_INVALID: return "invalid argument";
    case NXM_E_CUDA: return "CUDA runtime error";
    case NXM_E_CAPACITY: return "more active grid blocks than the grid capacity";
    case NXM_E_HASH_FULL: return "grid block hash map full";
    case NXM_E_NO_DEVICE: return "no sm_100 CUDA device available";
    case NXM_E_UNSUPPORTED: return "unsupported feature";
    case NXM_E_OOM: return "device out of memory";
    default: return "unknown error";
    }
}

int nxm_pipeline_create(nxm_pipeline** out) {
    if (!out) return NXM_E_INVALID;
    *out = nullptr;
    int dev = 0, sms = 0;
    if (!device_ok(&dev, &sms)) return NXM_E_NO_DEVICE;
    nxm_pipeline* p = new (std::nothrow) nxm_pipeline();
    if (!p) return NXM_E_OOM;
    p->device = dev;
    p->sm_count = sms;
    *out = p;
    return NXM_OK;
}

void nxm_pipeline_destroy(nxm_pipeline* p) { delete p; }

int nxm_state_create(const nxm_capacities* caps, nxm_state** out) {
    if (!out) return NXM_E_INVALID;
    *out = nullptr;
    int dev = 0, sms = 0;
    if (!device_ok(&dev, &sms)) return NXM_E_NO_DEVICE;
    nxm_capacities c = caps ? *caps : nxm_capacities{32768u, 65536u};
    nxm_state* s = new (std::nothrow) nxm_state();
    if (!s) return NXM_E_OOM;
    s->device = dev;
    s->sm_count = sms;
    int rc = NXM_OK;
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) rc = NXM_E_CUDA;
    if (!rc) {
        cudaMemPoolProps pp{};
        pp.allocType = cudaMemAllocationTypePinned;
        pp.handleTypes = cudaMemHandleTypeNone;
        pp.location.type = cudaMemLocationTypeDevice;
        pp.location.id = dev;
        uint64_t keep = UINT64_MAX;
        if (cudaMemPoolCreate(&s->pool, &pp) != cudaSuccess ||
            cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess)
            rc = NXM_E_CUDA;
    }
    if (!rc && dalloc(&s->d_params, 1) != cudaSuccess) rc = NXM_E_OOM;
    if (!rc && dalloc(&s->d_counters, 1) != cudaSuccess) rc = NXM_E_OOM;
    if (!rc && cudaMallocHost(reinterpret_cast<void**>(&s->h_counters), sizeof(Counters)) != cudaSuccess) rc = NXM_E_OOM;
    if (!rc && dalloc(&s->d_colliders, MAX_COLLIDERS) != cudaSuccess) rc = NXM_E_OOM;
    s->col_cap = MAX_COLLIDERS;
    if (!rc && cudaMemsetAsync(s->d_counters, 0, sizeof(Counters), s->stream) != cudaSuccess) rc = NXM_E_CUDA;
    if (!rc) rc = alloc_grid(s, c.grid_size);
    if (!rc) rc = reserve_particles(s, std::max<uint32_t>(c.particles_capacity, 1));
    if (!rc) rc = sync_params(s);
    if (rc) {
        nxm_state_destroy(s);
        (void)cudaGetLastError();
        return rc;
    }
    *out = s;
    return NXM_OK;
}

void nxm_state_destroy(nxm_state* s) {
    if (!s) return;
    if (s->stream) cudaStreamSynchronize(s->stream);
    invalidate_graph(s);
    free_grid(s);
    free_particles(s);
    dfree(s->d_materials); dfree(s->d_colliders); dfree(s->d_tris); dfree(s->d_bvh); dfree(s->d_scene_cols); dfree(s->d_vel6); dfree(s->d_params); dfree(s->d_counters);
    dfree(s->d_pack); dfree(s->d_offsets);
    dfree(s->d_rp_local); dfree(s->d_rp_world); dfree(s->d_rp_need); dfree(s->d_rp_sorted);
    dfree(s->d_render); dfree(s->d_palette);
    if (s->h_vel6) cudaFreeHost(s->h_vel6);
    if (s->h_status) cudaFreeHost(s->h_status);
    if (s->h_poll) cudaFreeHost(s->h_poll);
    if (s->poll_done) cudaEventDestroy(s->poll_done);
    if (s->stg) cudaFreeHost(s->stg);
    free_retired_rings(s);
    for (const auto& sp : s->stg_live) cudaEventDestroy(sp.done);
    for (const auto& f : s->fences) cudaEventDestroy(f.second);
    for (cudaEvent_t e : s->event_pool) cudaEventDestroy(e);
    for (cudaEvent_t e : s->vel_done)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : s->status_done)
        if (e) cudaEventDestroy(e);
    if (s->h_counters) cudaFreeHost(s->h_counters);
    if (s->pool) cudaMemPoolDestroy(s->pool);  // after d_pack, its last allocation, was freed above
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

int nxm_state_set_simulation_params(nxm_state* s, const nxm_simulation_params* p) {
    if (!s || !p) return NXM_E_INVALID;
    if (!(p->dt > 0.f)) return NXM_E_INVALID;
    std::memcpy(s->gravity, p->gravity, sizeof(s->gravity));
    s->base_dt = p->dt;
    s->dt = p->dt;
    s->params_dirty = true;
    return NXM_OK;
}

int nxm_state_write_substep_params(nxm_state* s, uint32_t num_substeps) {
    if (!s) return NXM_E_INVALID;
    s->dt = s->base_dt / (float)std::max<uint32_t>(num_substeps, 1u);
    s->params_dirty = true;
    return NXM_OK;
}

int nxm_state_set_cell_width(nxm_state* s, float cell_width, uint32_t grid_capacity) {
    if (!s || !(cell_width > 0.f) || grid_capacity == 0 || grid_capacity > (1u << 26)) return NXM_E_INVALID;
    s->dx = cell_width;
    int rc = alloc_grid(s, grid_capacity);
    if (rc) return rc;
    rc = rebuild_rigid_particles(s);  // sampled at the cell width
    if (rc) return rc;
    NXM_TRY(cudaStreamSynchronize(s->stream));
    s->params_dirty = true;
    return invalidate_codes(s);
}

int nxm_state_set_colliders(nxm_state* s, const nxm_collider* cols, uint32_t ncol, const float* tri, uint32_t ntri) {
    if (!s) return NXM_E_INVALID;
    if (s->scene_blocks) return NXM_E_INVALID;  // batched scenes bring their own colliders
    if (ncol > (uint32_t)MAX_COLLIDERS) return NXM_E_INVALID;
    if (ncol && !cols) return NXM_E_INVALID;
    std::vector<DevCollider> dc(ncol);
    for (uint32_t i = 0; i < ncol; ++i) {
        int rc = collider_from_abi(cols[i], tri, ntri, 0, dc[i]);
        if (rc) return rc;
    }
    return install_colliders(s, dc, tri);
}

int nxm_state_set_collider_velocity(nxm_state* s, uint32_t index, const float linvel[3], const float angvel[3]) {
    if (!s || !linvel || !angvel || index >= s->colliders.size()) return NXM_E_INVALID;
    // the values travel as a kernel argument: ordered on the stream, no host wait
    const Vel6 v{{linvel[0], linvel[1], linvel[2], angvel[0], angvel[1], angvel[2]}};
    k_set_velocity<<<1, 32, 0, s->stream>>>(s->d_colliders, index, v);
    s->launches += 1;
    NXM_TRY(cudaGetLastError());
    return NXM_OK;
}

int nxm_state_set_collider_velocities(nxm_state* s, uint32_t first, uint32_t count, const float* vel6) {
    if (!s || (count && !vel6) || first > s->colliders.size() || count > s->colliders.size() - first)
        return NXM_E_INVALID;
    if (count == 0) return NXM_OK;
    const size_t need = 6 * (size_t)count;
    if (need > s->vel_cap) {
        NXM_TRY(cudaStreamSynchronize(s->stream));  // the old slots may still be read
        dfree(s->d_vel6);
        if (s->h_vel6) cudaFreeHost(s->h_vel6);
        s->h_vel6 = nullptr;
        s->vel_cap = 0;
        NXM_TRY(dalloc(&s->d_vel6, need * nxm_state::kVelSlots));
        NXM_TRY(cudaMallocHost(reinterpret_cast<void**>(&s->h_vel6), 4 * need * nxm_state::kVelSlots));
        for (cudaEvent_t& e : s->vel_done)
            if (!e) NXM_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        s->vel_cap = need;
    }
    // copy into a pinned slot (its previous copy, kVelSlots calls ago, has run),
    // then a truly asynchronous transfer: the caller's array is free on return
    const int slot = s->vel_slot;
    s->vel_slot = (slot + 1) % nxm_state::kVelSlots;
    NXM_TRY(cudaEventSynchronize(s->vel_done[slot]));
    float* h = s->h_vel6 + s->vel_cap * slot;
    float* d = s->d_vel6 + s->vel_cap * slot;
    std::memcpy(h, vel6, 4 * need);
    NXM_TRY(cudaMemcpyAsync(d, h, 4 * need, cudaMemcpyHostToDevice, s->stream));
    NXM_TRY(cudaEventRecord(s->vel_done[slot], s->stream));
    k_set_velocities<<<(count + 127) / 128, 128, 0, s->stream>>>(s->d_colliders, d, first, count);
    s->launches += 1;
    NXM_TRY(cudaGetLastError());
    return NXM_OK;
}

int nxm_state_read_collider_pose(nxm_state* s, uint32_t index, float out[7]) {
    if (!s || !out || index >= s->colliders.size()) return NXM_E_INVALID;
    DevCollider c;
    NXM_TRY(cudaMemcpyAsync(&c, s->d_colliders + index, sizeof(c), cudaMemcpyDeviceToHost, s->stream));
    NXM_TRY(cudaStreamSynchronize(s->stream));
    std::memcpy(out, c.rot, 16);
    std::memcpy(out + 4, c.tra, 12);
    return NXM_OK;
}

int nxm_state_set_use_cpic(nxm_state* s, int enabled) {
    if (!s) return NXM_E_INVALID;
    if (enabled) {
        int rc = canonicalize(s);  // CPIC steps in place, in id order
        if (rc) return rc;
        rc = alloc_cpic_grid(s);
        if (rc) return rc;
    }
    if (s->use_cpic != (enabled != 0)) invalidate_graph(s);
    s->use_cpic = enabled != 0;
    s->params_dirty = true;
    return rebuild_rigid_particles(s);
}

// ---- render data (headless prep_readback) -----------------------------------

static_assert(sizeof(nxm_readback_data) == 96, "ReadbackData layout");
static_assert(NXM_RENDER_DEFAULT == RENDER_DEFAULT && NXM_RENDER_VOLUME == RENDER_VOLUME &&
                  NXM_RENDER_VELOCITY == RENDER_VELOCITY && NXM_RENDER_PHASE == RENDER_PHASE &&
                  NXM_RENDER_CDF_NORMALS == RENDER_CDF_NORMALS && NXM_RENDER_CDF_DISTANCES == RENDER_CDF_DISTANCES &&
                  NXM_RENDER_CDF_SIGNS == RENDER_CDF_SIGNS,
              "render modes");

// GpuReadbackData::DEFAULT_GROUP_COLORS (src_mpm/solver/prep_readback.rs).
static const float kDefaultPalette[6][4] = {
    {124.0f / 255.0f, 144.0f / 255.0f, 1.0f, 1.0f},          {8.0f / 255.0f, 144.0f / 255.0f, 1.0f, 1.0f},
    {124.0f / 255.0f, 7.0f / 255.0f, 1.0f, 1.0f},            {124.0f / 255.0f, 144.0f / 255.0f, 7.0f / 255.0f, 1.0f},
    {200.0f / 255.0f, 37.0f / 255.0f, 1.0f, 1.0f},           {124.0f / 255.0f, 230.0f / 255.0f, 25.0f / 255.0f, 1.0f}};

// Uploads the palette (null or empty: the default one) and fills `in`.
static int render_source(nxm_state* s, uint32_t mode, const float* palette, uint32_t num_groups, RenderSrc& in) {
    if (!palette || num_groups == 0) {
        palette = &kDefaultPalette[0][0];
        num_groups = 6;
    }
    if (num_groups > s->palette_cap) {
        NXM_TRY(cudaStreamSynchronize(s->stream));
        dfree(s->d_palette);
        NXM_TRY(dalloc(&s->d_palette, num_groups));
        s->palette_cap = num_groups;
    }
    NXM_TRY(cudaMemcpyAsync(s->d_palette, palette, sizeof(float4) * num_groups, cudaMemcpyHostToDevice, s->stream));
    in.kin = s->kin;
    in.def = s->def;
    in.pcdf = s->d_pcdf;
    in.pid = s->permuted ? s->pid : nullptr;
    in.n = s->n;
    in.mode = mode;
    in.palette = s->d_palette;
    in.num_groups = num_groups;
    in.dx = s->dx;
    in.dt = s->dt;
    in.sm_count = s->sm_count;
    return NXM_OK;
}

static int render_scratch(nxm_state* s, size_t records) {
    if (6 * records <= s->render_cap) return NXM_OK;
    NXM_TRY(cudaStreamSynchronize(s->stream));
    dfree(s->d_render);
    NXM_TRY(dalloc(&s->d_render, 6 * records));
    s->render_cap = 6 * records;
    return NXM_OK;
}

int nxm_prep_readback(nxm_state* s, uint32_t mode, const float* palette, uint32_t num_groups, nxm_readback_data* out) {
    if (!s || (s->n && !out)) return NXM_E_INVALID;
    if (s->n == 0) return NXM_OK;
    RenderSrc in{};
    int rc = render_source(s, mode, palette, num_groups, in);
    if (rc) return rc;
    rc = render_scratch(s, s->n);
    if (rc) return rc;
    launch_prep_readback(in, s->d_render, s->stream);
    s->launches += 1;
    NXM_TRY(cudaGetLastError());
    NXM_TRY(cudaMemcpyAsync(out, s->d_render, sizeof(nxm_readback_data) * s->n, cudaMemcpyDeviceToHost, s->stream));
    NXM_TRY(cudaStreamSynchronize(s->stream));
    return NXM_OK;
}

int nxm_prep_render(nxm_state* s, uint32_t mode, const float* palette, uint32_t num_groups, float* positions,
                    float* deformations, float* colors) {
    if (!s || (s->n && (!positions || !deformations || !colors))) return NXM_E_INVALID;
    if (reinterpret_cast<uintptr_t>(colors) % 16 != 0) return NXM_E_INVALID;
    if (s->n == 0) return NXM_OK;
    RenderSrc in{};
    int rc = render_source(s, mode, palette, num_groups, in);
    if (rc) return rc;
    launch_prep_render(in, positions, deformations, colors, s->stream);
    s->launches += 1;
    NXM_TRY(cudaGetLastError());
    return NXM_OK;
}

int nxm_prep_readback_rigid(nxm_state* s, const float* colors, const float* palette, uint32_t num_groups,
                            nxm_readback_data* out) {
    if (!s || (s->nrp && !out)) return NXM_E_INVALID;
    if (s->nrp == 0) return NXM_OK;
    RenderSrc in{};
    int rc = render_source(s, RENDER_DEFAULT, palette, num_groups, in);
    if (rc) return rc;
    rc = render_scratch(s, (size_t)s->nrp * (colors ? 2 : 1));
    if (rc) return rc;
    const float4* d_colors = nullptr;
    if (colors) {  // per rigid particle base colors, staged after the records
        NXM_TRY(cudaMemcpyAsync(s->d_render + 6 * (size_t)s->nrp, colors, sizeof(float4) * s->nrp,
                                cudaMemcpyHostToDevice, s->stream));
        d_colors = s->d_render + 6 * (size_t)s->nrp;
    }
    launch_prep_readback_rigid(in, s->d_rp_world, s->nrp, d_colors, s->d_render, s->stream);
    s->launches += 1;
    NXM_TRY(cudaGetLastError());
    NXM_TRY(cudaMemcpyAsync(out, s->d_render, sizeof(nxm_readback_data) * s->nrp, cudaMemcpyDeviceToHost, s->stream));
    NXM_TRY(cudaStreamSynchronize(s->stream));
    return NXM_OK;
}

int nxm_state_num_rigid_particles(const nxm_state* s, uint32_t* count) {
    if (!s || !count) return NXM_E_INVALID;
    *count = s->nrp;
    return NXM_OK;
}

int nxm_read_rigid_particles(nxm_state* s, float* out) {
    if (!s || (s->nrp && !out)) return NXM_E_INVALID;
    for (uint32_t i = 0; i < s->nrp; ++i) {
        const float4& r = s->rp_host[i];
        const uint32_t word = f_bits(r.w);
        const uint32_t col = word >> kRigidTriBits;
        float* o = out + 5 * (size_t)i;
        o[0] = r.x; o[1] = r.y; o[2] = r.z;
        o[3] = bits_f(col);
        o[4] = bits_f((word & kRigidTriMask) - s->tri_base[col]);
    }
    return NXM_OK;
}

int nxm_read_cdf(nxm_state* s, float* out) {
    if (!s) return NXM_E_INVALID;
    static const int off[8] = {0, 1, 2, 3, 4, 5, 6, 7};
    if (s->permuted) return NXM_E_INVALID;  // the fields are id-indexed; CPIC keeps id order
    return pack_read(s, s->d_pcdf, 48, off, 8, out);
}

int nxm_state_set_deterministic(nxm_state* s, int enabled) {
    if (!s) return NXM_E_INVALID;
    if (enabled) {  // the deterministic step works in place, in id order
        int rc = canonicalize(s);
        if (rc) return rc;
    }
    if (s->deterministic != (enabled != 0)) invalidate_graph(s);
    s->deterministic = enabled != 0;
    return NXM_OK;
}

int nxm_particles_append_soa(nxm_state* s, const nxm_particles_soa* p, uint32_t count) {
    if (!s) return NXM_E_INVALID;
    if (s->scene_blocks) return NXM_E_INVALID;  // in scene mode particles change through the scene calls
    return upload_particles(s, p, count);
}

int nxm_particles_append(nxm_state* s, const nxm_particle* particles, uint32_t count) {
    if (!s || (count && !particles)) return NXM_E_INVALID;
    if (s->scene_blocks) return NXM_E_INVALID;  // in scene mode particles change through the scene calls
    if (count == 0) return NXM_OK;
    std::vector<float> pos(3 * (size_t)count), vel(3 * (size_t)count), F(9 * (size_t)count), A(9 * (size_t)count);
    std::vector<float> vgd(count), v0(count), rad(count), mass(count), damp(count), phase(count), bf(count);
    std::vector<uint32_t> gid(count), en(count), fx(count);
    std::vector<nxm_particle_model> models(count);
    for (uint32_t i = 0; i < count; ++i) {
        const nxm_particle& q = particles[i];
        std::memcpy(&pos[3 * (size_t)i], q.position, 12);
        std::memcpy(&vel[3 * (size_t)i], q.velocity, 12);
        std::memcpy(&F[9 * (size_t)i], q.def_grad, 36);
        std::memcpy(&A[9 * (size_t)i], q.affine, 36);
        vgd[i] = q.vel_grad_det; v0[i] = q.init_volume; rad[i] = q.init_radius; mass[i] = q.mass;
        damp[i] = q.damping; phase[i] = q.phase; bf[i] = q.boundary_friction;
        gid[i] = q.group_id; en[i] = q.enabled; fx[i] = q.fixed; models[i] = q.model;
    }
    nxm_particles_soa soa{pos.data(), vel.data(), F.data(), A.data(), vgd.data(), v0.data(), rad.data(), mass.data(),
                          damp.data(), phase.data(), bf.data(), gid.data(), en.data(), fx.data(), models.data()};
    return upload_particles(s, &soa, count);
}

uint32_t nxm_particles_len(const nxm_state* s) { return s ? s->n : 0u; }

// ---- batched scenes ------------------------------------------------------------

static int floor_div_i(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

int nxm_state_enable_scenes(nxm_state* s, uint32_t scene_blocks) {
    if (!s || s->n != 0 || !s->colliders.empty()) return NXM_E_INVALID;
    if (scene_blocks != 0 && (scene_blocks < 8 || scene_blocks > 512)) return NXM_E_INVALID;
    dfree(s->d_scene_cols);
    s->scenes.clear();
    s->scene_blocks = scene_blocks;
    if (scene_blocks) {
        const int S = (int)scene_blocks, M = S / 8;
        s->scene_margin = M;
        // cells whose key region [c S - M, c S + S - M) lies inside the packed-key range
        const int lo[3] = {-1023, -511, -1023}, hi[3] = {1024, 512, 1024};
        size_t total = 1;
        for (int k = 0; k < 3; ++k) {
            const int cmin = -floor_div_i(-(lo[k] + M), S);  // ceil((lo + M) / S)
            const int cmax = floor_div_i(hi[k] + 1 + M - S, S);
            s->scene_cmin[k] = cmin;
            s->scene_cells[k] = (uint32_t)std::max(0, cmax - cmin + 1);
            total *= s->scene_cells[k];
        }
        s->scenes.assign(total, nxm_state::Scene{});
        NXM_TRY(dalloc(&s->d_scene_cols, total));
        NXM_TRY(cudaMemset(s->d_scene_cols, 0, sizeof(uint2) * total));
    }
    invalidate_graph(s);
    s->params_dirty = true;
    return NXM_OK;
}

uint32_t nxm_scene_capacity(const nxm_state* s) { return s ? (uint32_t)s->scenes.size() : 0u; }

// Collider table of the live scenes, in scene-slot order, and each slot's range.
static int rebuild_scene_colliders(nxm_state* s) {
    std::vector<DevCollider> dc;
    std::vector<float> tri;
    std::vector<uint2> ranges(s->scenes.size(), make_uint2(0u, 0u));
    for (size_t i = 0; i < s->scenes.size(); ++i) {
        const nxm_state::Scene& sc = s->scenes[i];
        if (!sc.live) continue;
        const uint32_t toff = (uint32_t)(tri.size() / 9);
        ranges[i] = make_uint2((uint32_t)dc.size(), (uint32_t)sc.cols.size());
        for (const nxm_collider& c : sc.cols) {
            DevCollider d;
            int rc = collider_from_abi(c, sc.tri.data(), (uint32_t)(sc.tri.size() / 9), toff, d);
            if (rc) return rc;
            d.scene = (uint32_t)i;
            dc.push_back(d);
        }
        tri.insert(tri.end(), sc.tri.begin(), sc.tri.end());
    }
    NXM_TRY(upload_async(s, s->d_scene_cols, ranges.data(), sizeof(uint2) * ranges.size()));
    return install_colliders(s, dc, tri.data());
}

int nxm_scene_add(nxm_state* s, const nxm_particles_soa* particles, uint32_t count, const nxm_collider* colliders,
                  uint32_t num_colliders, const float* tri_vertices, uint32_t num_triangles, uint32_t* scene) {
    if (!s || !scene || !s->scene_blocks || (count && (!particles || !particles->position))) return NXM_E_INVALID;
    if (num_colliders > (uint32_t)MAX_COLLIDERS || (num_colliders && !colliders)) return NXM_E_INVALID;
    for (uint32_t i = 0; i < num_colliders; ++i) {
        DevCollider d;
        int rc = collider_from_abi(colliders[i], tri_vertices, num_triangles, 0, d);
        if (rc) return rc;
    }
    // every particle's block (and its +1 neighbours) must stay inside the scene's
    // key region: the floor of a coordinate / block width grows with the
    // coordinate, so the extremes (and no NaN) decide it; found on host threads
    const float bw = 4.0f * s->dx;
    const int M = s->scene_margin, S = (int)s->scene_blocks;
    if (count) {
        const float* x = particles->position;
        const size_t total = 3 * (size_t)count;
        const unsigned hw = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
        const unsigned nt = total < (size_t(1) << 18) ? 1u : hw;
        std::vector<std::array<float, 7>> ext(nt);  // per thread: min xyz, max xyz, NaN seen
        auto scan = [&](unsigned t) {
            std::array<float, 7> e{INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY, 0.f};
            const size_t lo = count * (size_t)t / nt, hi = count * (size_t)(t + 1) / nt;
            for (size_t i = lo; i < hi; ++i)
                for (int a = 0; a < 3; ++a) {
                    const float v = x[3 * i + a];
                    if (v != v) e[6] = 1.f;
                    e[a] = std::min(e[a], v);
                    e[3 + a] = std::max(e[3 + a], v);
                }
            ext[t] = e;
        };
        if (nt == 1) {
            scan(0);
        } else {
            std::vector<std::thread> th;
            for (unsigned t = 0; t < nt; ++t) th.emplace_back(scan, t);
            for (auto& t : th) t.join();
        }
        for (const auto& e : ext) {
            if (e[6] != 0.f) return NXM_E_INVALID;
            for (int a = 0; a < 3; ++a) {
                if (e[a] > e[3 + a]) continue;  // this thread saw no particle
                const float blo = std::floor(e[a] / bw), bhi = std::floor(e[3 + a] / bw);
                if (!(blo >= (float)(1 - M) && bhi <= (float)(S - M - 3))) return NXM_E_INVALID;
            }
        }
    }
    uint32_t slot = 0;
    while (slot < s->scenes.size() && s->scenes[slot].live) ++slot;
    if (slot == s->scenes.size()) return NXM_E_CAPACITY;
    const uint32_t first = s->n;
    int rc = count ? upload_particles(s, particles, count) : NXM_OK;
    if (rc) return rc;
    if (count) {
        k_fill<<<grid_for_n(s, count), 256, 0, s->stream>>>(s->d_pscene + first, slot, count);
        s->launches += 1;
        NXM_TRY(cudaGetLastError());
    }
    nxm_state::Scene& sc = s->scenes[slot];
    sc.live = true;
    sc.first = first;
    sc.count = count;
    sc.cols.assign(colliders, colliders + num_colliders);
    sc.tri.assign(tri_vertices ? tri_vertices : nullptr,
                  tri_vertices ? tri_vertices + 9 * (size_t)num_triangles : nullptr);
    rc = rebuild_scene_colliders(s);
    if (rc) return rc;
    *scene = slot;
    return NXM_OK;
}

int nxm_scene_remove(nxm_state* s, const uint32_t* scenes, uint32_t count) {
    if (!s || (count && !scenes) || !s->scene_blocks) return NXM_E_INVALID;
    std::vector<uint2> ranges;
    std::vector<uint32_t> ids(scenes, scenes + count);
    std::sort(ids.begin(), ids.end());
    ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
    for (uint32_t id : ids)
        if (id >= s->scenes.size() || !s->scenes[id].live) return NXM_E_INVALID;
    for (uint32_t id : ids) ranges.push_back(make_uint2(s->scenes[id].first, s->scenes[id].first + s->scenes[id].count));
    int rc = remove_id_ranges(s, ranges);
    if (rc) return rc;
    for (uint32_t id : ids) s->scenes[id] = nxm_state::Scene{};
    for (nxm_state::Scene& sc : s->scenes) {  // ids after a removed range shift down by its length
        if (!sc.live) continue;
        uint32_t shift = 0;
        for (uint2 r : ranges)
            if (r.x < sc.first) shift += r.y - r.x;
        sc.first -= shift;
    }
    return rebuild_scene_colliders(s);
}

int nxm_scene_range(const nxm_state* s, uint32_t scene, uint32_t* first, uint32_t* count) {
    if (!s || !first || !count || scene >= s->scenes.size() || !s->scenes[scene].live) return NXM_E_INVALID;
    *first = s->scenes[scene].first;
    *count = s->scenes[scene].count;
    return NXM_OK;
}

int nxm_scene_set_collider_velocity(nxm_state* s, uint32_t scene, uint32_t index, const float linvel[3],
                                    const float angvel[3]) {
    if (!s || scene >= s->scenes.size() || !s->scenes[scene].live || index >= s->scenes[scene].cols.size())
        return NXM_E_INVALID;
    uint32_t global = 0;
    for (uint32_t i = 0; i < scene; ++i)
        if (s->scenes[i].live) global += (uint32_t)s->scenes[i].cols.size();
    return nxm_state_set_collider_velocity(s, global + index, linvel, angvel);
}

int nxm_read_positions_range(nxm_state* s, uint32_t first, uint32_t count, float* out) {
    if (!s) return NXM_E_INVALID;
    static const int off[3] = {0, 1, 2};
    return pack_read_range(s, s->kin, sizeof(PKin), off, 3, first, count, out);
}

// ---- particle chunks (NexusState, src/state.rs:665-774) ---------------------

int nxm_chunk_add(nxm_state* s, const nxm_particle* particles, uint32_t count, uint32_t* chunk) {
    if (!s || !chunk || s->scene_blocks) return NXM_E_INVALID;
    if (!s->chunks_used) {
        s->slot2chunk.assign(s->n, NONE);
        s->chunks_used = true;
    }
    const uint32_t n0 = s->n;
    int rc = nxm_particles_append(s, particles, count);
    if (rc) return rc;
    const uint32_t id = s->next_chunk++;
    std::fill(s->slot2chunk.begin() + n0, s->slot2chunk.end(), id);
    s->chunks[id] = count;
    *chunk = id;
    return NXM_OK;
}

int nxm_chunk_extend(nxm_state* s, uint32_t chunk, const nxm_particle* particles, uint32_t count) {
    if (!s) return NXM_E_INVALID;
    auto it = s->chunks.find(chunk);
    if (it == s->chunks.end()) return NXM_E_INVALID;
    const uint32_t n0 = s->n;
    int rc = nxm_particles_append(s, particles, count);
    if (rc) return rc;
    std::fill(s->slot2chunk.begin() + n0, s->slot2chunk.end(), chunk);
    it->second += count;
    return NXM_OK;
}

// Slots of `chunk`, highest first, at most `limit`.
static std::vector<uint32_t> chunk_slots_desc(const nxm_state* s, uint32_t chunk, size_t limit) {
    std::vector<uint32_t> slots;
    for (uint32_t i = s->n; i-- > 0 && slots.size() < limit;)
        if (s->slot2chunk[i] == chunk) slots.push_back(i);
    return slots;
}

int nxm_chunk_remove(nxm_state* s, uint32_t chunk) {
    if (!s) return NXM_E_INVALID;
    auto it = s->chunks.find(chunk);
    if (it == s->chunks.end()) return NXM_E_INVALID;
    std::vector<uint32_t> slots = chunk_slots_desc(s, chunk, s->n);
    int rc = nxm_particles_swap_remove(s, slots.data(), (uint32_t)slots.size(), nullptr, nullptr);
    if (rc) return rc;
    s->chunks.erase(chunk);
    return NXM_OK;
}

int nxm_chunk_remove_particles(nxm_state* s, uint32_t chunk, uint32_t count, uint32_t* removed) {
    if (!s) return NXM_E_INVALID;
    auto it = s->chunks.find(chunk);
    if (it == s->chunks.end()) return NXM_E_INVALID;
    std::vector<uint32_t> slots = chunk_slots_desc(s, chunk, count);
    int rc = nxm_particles_swap_remove(s, slots.data(), (uint32_t)slots.size(), nullptr, nullptr);
    if (rc) return rc;
    it->second -= std::min<uint32_t>(it->second, (uint32_t)slots.size());
    if (removed) *removed = (uint32_t)slots.size();
    return NXM_OK;
}

int nxm_chunk_len(const nxm_state* s, uint32_t chunk, uint32_t* len) {
    if (!s || !len) return NXM_E_INVALID;
    auto it = s->chunks.find(chunk);
    if (it == s->chunks.end()) return NXM_E_INVALID;
    *len = it->second;
    return NXM_OK;
}

int nxm_chunk_of_particles(const nxm_state* s, uint32_t* out) {
    if (!s || (s->n && !out)) return NXM_E_INVALID;
    if (!s->chunks_used) std::fill(out, out + s->n, NONE);
    else std::copy(s->slot2chunk.begin(), s->slot2chunk.end(), out);
    return NXM_OK;
}

int nxm_particles_swap_remove(nxm_state* s, const uint32_t* slots, uint32_t count, uint32_t* remaps,
                              uint32_t* num_remaps) {
    if (!s || (count && !slots)) return NXM_E_INVALID;
    if (s->scene_blocks) return NXM_E_INVALID;  // in scene mode particles change through the scene calls
    int rc = canonicalize(s);
    if (rc) return rc;
    s->sort_pid = nullptr;
    std::vector<uint32_t> t(slots, slots + count);
    std::sort(t.begin(), t.end(), [](uint32_t a, uint32_t b) { return a > b; });
    t.erase(std::unique(t.begin(), t.end()), t.end());
    while (!t.empty() && t.front() >= s->n) t.erase(t.begin());  // out-of-range slots are ignored
    if (t.empty()) {
        if (num_remaps) *num_remaps = 0;
        return NXM_OK;
    }
    const uint32_t n0 = s->n, n1 = n0 - (uint32_t)t.size();
    // GpuParticles::swap_remove (src_mpm/solver/particle.rs:571-631): slots in
    // descending order, each replaced by the current last particle; the remap
    // list reports those moves in that order.
    uint32_t nr = 0, n = n0;
    for (uint32_t slot : t) {
        const uint32_t last = n - 1;
        if (slot != last) {
            if (s->chunks_used) s->slot2chunk[slot] = s->slot2chunk[last];
            if (remaps && nr < count) {
                remaps[2 * nr] = last;
                remaps[2 * nr + 1] = slot;
            }
            ++nr;
        }
        --n;
    }
    // The same result in one pass on the device: the i-th surviving particle
    // at or above n1 (descending) lands in the i-th removed slot below n1
    // (descending).  Sources are all >= n1 and destinations < n1.
    std::vector<uint2> pairs;
    {
        std::vector<uint32_t> dst;  // removed slots below n1, descending
        for (uint32_t slot : t)
            if (slot < n1) dst.push_back(slot);
        size_t k = 0;
        auto removed = t.begin();  // descending
        for (uint32_t src = n0; src-- > n1;) {
            while (removed != t.end() && *removed > src) ++removed;
            if (removed != t.end() && *removed == src) continue;  // removed itself
            pairs.push_back(make_uint2(dst[k++], src));
        }
    }
    if (!pairs.empty()) {
        uint2* d_pairs = nullptr;
        NXM_TRY(dalloc(&d_pairs, pairs.size()));
        cudaError_t e = cudaMemcpyAsync(d_pairs, pairs.data(), sizeof(uint2) * pairs.size(), cudaMemcpyHostToDevice,
                                        s->stream);
        if (e == cudaSuccess) {
            k_move_records<<<grid_for_n(s, (uint32_t)pairs.size()), 256, 0, s->stream>>>(s->kin, s->def, s->pstate,
                                                                                        s->d_pcdf, d_pairs,
                                                                                        (uint32_t)pairs.size());
            s->launches += 1;
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        cudaFree(d_pairs);
        NXM_TRY(e);
    }
    if (s->chunks_used) s->slot2chunk.resize(n1);
    s->n = n1;
    if (num_remaps) *num_remaps = nr;
    s->params_dirty = true;
    return invalidate_codes(s);
}

int nxm_particles_shift_remove(nxm_state* s, uint32_t start, uint32_t end) {
    if (!s || start > end || end > s->n) return NXM_E_INVALID;
    if (s->scene_blocks) return NXM_E_INVALID;  // in scene mode particles change through the scene calls
    if (start == end) return NXM_OK;
    return remove_id_ranges(s, {make_uint2(start, end)});
}

int nxm_step(nxm_pipeline* pipeline, nxm_state* s, nxm_timestamps* ts) {
    if (!pipeline || !s) return NXM_E_INVALID;
    int rc = ensure_ready(s);
    if (rc) return rc;
    if (s->n == 0) return NXM_OK;
    rc = prepare_reorder(s);
    if (rc) return rc;
    if (ts) {
        cudaEvent_t ev[5];
        for (auto& e : ev) NXM_TRY(cudaEventCreate(&e));
        int k = enqueue_step(s, s->stream, ev);
        s->launches += (uint64_t)k;
        finish_step(s);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaEventSynchronize(ev[4]);
        if (e == cudaSuccess) {
            cudaEventElapsedTime(&ts->sort_ms, ev[0], ev[1]);
            cudaEventElapsedTime(&ts->p2g_ms, ev[1], ev[2]);
            cudaEventElapsedTime(&ts->grid_update_ms, ev[2], ev[3]);
            cudaEventElapsedTime(&ts->g2p_ms, ev[3], ev[4]);
            cudaEventElapsedTime(&ts->total_ms, ev[0], ev[4]);
        }
        for (auto& x : ev) cudaEventDestroy(x);
        return e == cudaSuccess ? NXM_OK : NXM_E_CUDA;
    }
    if (!s->graph_valid[s->parity]) {
        rc = build_graph(s);
        if (rc) return rc;
    }
    NXM_TRY(cudaGraphLaunch(s->graph[s->parity], s->stream));
    s->launches += (uint64_t)s->graph_kernels;
    finish_step(s);
    return NXM_OK;
}

int nxm_debug_sort(nxm_pipeline* pipeline, nxm_state* s, int with_p2g) {
    if (!pipeline || !s) return NXM_E_INVALID;
    int rc = ensure_ready(s);
    if (rc) return rc;
    if (s->n == 0) return NXM_OK;
    DevPtrs P = dev_ptrs(s);
    LaunchCfg c = launch_cfg(s);
    fast::launch_sort(P, c, /*with_extras=*/true, /*canonical=*/s->deterministic, s->stream);
    s->launches += (uint64_t)sort_launches(s->deterministic);
    s->sort_pid = s->permuted ? s->pid : nullptr;
    if (with_p2g) {
        if (s->deterministic) exact::launch_p2g_gather(P, c, s->stream);
        else fast::launch_p2g(P, c, s->stream);
        s->launches += 1;
    }
    NXM_TRY(cudaGetLastError());
    NXM_TRY(cudaStreamSynchronize(s->stream));
    return NXM_OK;
}

int nxm_debug_fail_allocation(int64_t after) {
    if (after < -1) return NXM_E_INVALID;
    g_alloc_fail_in.store(after);
    return NXM_OK;
}

int nxm_debug_copy_wait_timeout(nxm_state* s, uint32_t limit) {
    if (!s) return NXM_E_INVALID;
    fast::launch_copy_wait_timeout(s->d_counters, limit, s->stream);
    s->launches += 1;
    NXM_TRY(cudaGetLastError());
    return NXM_OK;
}

int nxm_state_estimate_timestep_bound(nxm_state* s, float* max_dt, uint32_t* bits) {
    if (!s || !max_dt) return NXM_E_INVALID;
    int rc = ensure_ready(s);
    if (rc) return rc;
    NXM_TRY(cudaMemsetAsync(reinterpret_cast<char*>(s->d_counters) + offsetof(Counters, dt_bound), 0xFF, 4,
                            s->stream));
    if (s->n) {
        exact::launch_timestep_bound(dev_ptrs(s), launch_cfg(s), s->stream);
        s->launches += 1;
        NXM_TRY(cudaGetLastError());
    }
    NXM_TRY(cudaMemcpyAsync(s->h_counters, s->d_counters, sizeof(Counters), cudaMemcpyDeviceToHost, s->stream));
    NXM_TRY(cudaStreamSynchronize(s->stream));
    const uint32_t b = s->h_counters->dt_bound;
    if (bits) *bits = b;
    *max_dt = (float)b / 1.0e12f;
    return NXM_OK;
}

int nxm_simulate_frame(nxm_pipeline* pipeline, nxm_state* s, uint32_t min_substeps, uint32_t max_substeps,
                       uint32_t* substeps) {
    if (!pipeline || !s || max_substeps == 0 || min_substeps > max_substeps) return NXM_E_INVALID;
    float bound = 0.f;
    uint32_t bits = 0;
    int rc = nxm_state_estimate_timestep_bound(s, &bound, &bits);
    if (rc) return rc;
    uint32_t n = std::max<uint32_t>(min_substeps, 1u);
    if (bits == 0u) {
        n = max_substeps;  // a zero bound (a degenerate particle): as many substeps as allowed
    } else if (bits != 0xFFFFFFFFu) {  // 0xFFFFFFFF: no enabled particle, no constraint
        const double need = std::ceil((double)s->base_dt / ((double)bits / 1.0e12));
        if (need > (double)n) n = need >= (double)max_substeps ? max_substeps : (uint32_t)need;
    }
    n = std::min(n, max_substeps);
    rc = nxm_state_write_substep_params(s, n);
    if (rc) return rc;
    for (uint32_t i = 0; i < n; ++i) {
        rc = nxm_step(pipeline, s, nullptr);
        if (rc) return rc;
    }
    if (substeps) *substeps = n;
    return NXM_OK;
}

int nxm_synchronize(nxm_state* s) {
    if (!s) return NXM_E_INVALID;
    NXM_TRY(cudaStreamSynchronize(s->stream));
    free_retired_rings(s);
    uint32_t bits = 0;
    int rc = nxm_state_status(s, &bits, 0);
    if (rc) return rc;
    if (bits & NXM_STATUS_COPY_TIMEOUT) return NXM_E_CUDA;
    if (bits & NXM_STATUS_HASH_FULL) return NXM_E_HASH_FULL;
    if (bits & (NXM_STATUS_BLOCK_CAPACITY | NXM_STATUS_MISSING_BLOCK | NXM_STATUS_SORT_CAPACITY)) return NXM_E_CAPACITY;
    return NXM_OK;
}

int nxm_state_status_poll(nxm_state* s, uint32_t* bits, int* ready) {
    if (!s || !bits || !ready) return NXM_E_INVALID;
    if (!s->h_poll) {
        NXM_TRY(cudaHostAlloc(reinterpret_cast<void**>(&s->h_poll), sizeof(uint32_t), cudaHostAllocMapped));
        s->h_poll[0] = 0;
        NXM_TRY(cudaHostGetDevicePointer(reinterpret_cast<void**>(&s->h_poll_dev), s->h_poll, 0));
        NXM_TRY(cudaEventCreateWithFlags(&s->poll_done, cudaEventDisableTiming));
    }
    *bits = 0;
    *ready = 0;
    if (s->poll_outstanding) {
        const cudaError_t q = cudaEventQuery(s->poll_done);
        if (q == cudaErrorNotReady) {
            (void)cudaGetLastError();
            return NXM_OK;  // the last post has not run yet: no new one either
        }
        NXM_TRY(q);
        *bits = s->h_poll[0];
        *ready = 1;
        s->poll_outstanding = false;
    }
    k_post_status<<<1, 32, 0, s->stream>>>(s->d_counters, s->h_poll_dev);
    s->launches += 1;
    NXM_TRY(cudaGetLastError());
    NXM_TRY(cudaEventRecord(s->poll_done, s->stream));
    s->poll_outstanding = true;
    return NXM_OK;
}

int nxm_state_status_pipelined(nxm_state* s, uint32_t* bits) {
    if (!s || !bits) return NXM_E_INVALID;
    if (!s->h_status) {
        NXM_TRY(cudaHostAlloc(reinterpret_cast<void**>(&s->h_status), 2 * sizeof(uint32_t), cudaHostAllocMapped));
        s->h_status[0] = s->h_status[1] = 0;
        NXM_TRY(cudaHostGetDevicePointer(reinterpret_cast<void**>(&s->h_status_dev), s->h_status, 0));
        for (cudaEvent_t& e : s->status_done) NXM_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    const int cur = (int)(s->status_calls & 1u), prev = cur ^ 1;
    // slot `cur` was read by the previous call (after its write completed): free to be written again
    k_post_status<<<1, 32, 0, s->stream>>>(s->d_counters, s->h_status_dev + cur);
    s->launches += 1;
    NXM_TRY(cudaGetLastError());
    NXM_TRY(cudaEventRecord(s->status_done[cur], s->stream));
    *bits = 0;
    if (s->status_calls > 0) {
        NXM_TRY(cudaEventSynchronize(s->status_done[prev]));
        *bits = s->h_status[prev];
    }
    ++s->status_calls;
    return NXM_OK;
}

// ---- tickets ----------------------------------------------------------------
//
// A ticket marks the work queued on the state's stream so far; tickets
// complete in the order they were taken (one stream).

namespace {

// Retires the oldest fences: those already complete, and (wait) every one up
// to `upto`, waiting for it.
int retire_fences(nxm_state* s, uint64_t upto, bool wait) {
    while (!s->fences.empty()) {
        auto [t, e] = s->fences.front();
        if (wait && t <= upto) {
            NXM_TRY(cudaEventSynchronize(e));
        } else {
            const cudaError_t q = cudaEventQuery(e);
            if (q == cudaErrorNotReady) break;
            NXM_TRY(q);
        }
        s->done_ticket = t;
        s->event_pool.push_back(e);
        s->fences.pop_front();
    }
    if (wait && !s->stg_retired.empty()) free_retired_rings(s, /*drained=*/false);
    return NXM_OK;
}

}  // namespace

int nxm_state_fence(nxm_state* s, uint64_t* ticket) {
    if (!s || !ticket) return NXM_E_INVALID;
    cudaEvent_t e;
    NXM_TRY(take_event(s, &e));
    NXM_TRY(cudaEventRecord(e, s->stream));
    s->fences.emplace_back(s->next_ticket, e);
    *ticket = s->next_ticket++;
    int rc = retire_fences(s, 0, false);
    // a caller that never asks keeps at most 1024 events: wait for the oldest
    while (!rc && s->fences.size() > 1024u) rc = retire_fences(s, s->fences.front().first, true);
    return rc;
}

int nxm_state_ticket_done(nxm_state* s, uint64_t ticket, int* done) {
    if (!s || !done || ticket == 0 || ticket >= s->next_ticket) return NXM_E_INVALID;
    const int rc = retire_fences(s, 0, false);
    *done = ticket <= s->done_ticket;
    return rc;
}

int nxm_state_ticket_wait(nxm_state* s, uint64_t ticket) {
    if (!s || ticket == 0 || ticket >= s->next_ticket) return NXM_E_INVALID;
    return retire_fences(s, ticket, true);
}

int nxm_read_positions_range_async(nxm_state* s, uint32_t first, uint32_t count, float* out, uint64_t* ticket) {
    if (!s || !ticket) return NXM_E_INVALID;
    static const int off[3] = {0, 1, 2};
    const int rc = pack_read_range(s, s->kin, sizeof(PKin), off, 3, first, count, out, /*wait=*/false);
    if (rc) return rc;
    return nxm_state_fence(s, ticket);
}

// ---- autotuner ----------------------------------------------------------------
//
// nxm_state_autotune times the state's own steps under candidate launch
// shapes (coordinate descent over the knobs below, one knob at a time, the
// others held) and keeps the fastest; the decision is cached in a process-wide
// table keyed by the scene's density (particles per primary block, rounded
// down to a power of two) and its active scene count (rounded up to a power
// of two), which later states of the same kind apply with trial_steps = 0.

namespace {

struct TuneEntry {
    Tuning t;
    uint32_t fill;
    float ms_before, ms_after;
};
std::mutex g_tune_mutex;
std::map<uint64_t, TuneEntry> g_tune_table;

uint32_t floor_pow2(uint32_t v) { return v ? 1u << (31 - __builtin_clz(v)) : 0u; }

// The table key from the counters of the last step (false when no step has
// set them yet).
int tune_key(nxm_state* s, uint32_t* density, uint32_t* scenes, bool* known) {
    NXM_TRY(cudaMemcpyAsync(s->h_counters, s->d_counters, sizeof(Counters), cudaMemcpyDeviceToHost, s->stream));
    NXM_TRY(cudaStreamSynchronize(s->stream));
    *known = s->h_counters->num_primary > 0;
    const uint32_t nbp = std::max<uint32_t>(1u, std::min(s->h_counters->num_primary, s->h_counters->num_blocks));
    *density = floor_pow2(std::max<uint32_t>(1u, s->n / nbp));
    uint32_t live = 0;
    for (const auto& sc : s->scenes) live += sc.live ? 1u : 0u;
    *scenes = live ? next_pow2(live) : 0u;
    return NXM_OK;
}

void apply_tuning(nxm_state* s, const Tuning& t, uint32_t fill) {
    s->tuning = t;
    if (s->range_min_fill != fill) {
        s->range_min_fill = fill;
        s->params_dirty = true;
    }
    invalidate_graph(s);
}

// ms per step of `steps` graph steps after one untimed step (which captures
// the graph of the new shapes), CUDA events on the state's stream.
int time_steps(nxm_pipeline* pipe, nxm_state* s, uint32_t steps, float* ms) {
    int rc = nxm_step(pipe, s, nullptr);
    if (rc) return rc;
    cudaEvent_t a, b;
    NXM_TRY(cudaEventCreate(&a));
    NXM_TRY(cudaEventCreate(&b));
    NXM_TRY(cudaEventRecord(a, s->stream));
    for (uint32_t i = 0; i < steps && !rc; ++i) rc = nxm_step(pipe, s, nullptr);
    NXM_TRY(cudaEventRecord(b, s->stream));
    NXM_TRY(cudaEventSynchronize(b));
    float t = 0.f;
    cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *ms = t / (float)std::max<uint32_t>(steps, 1u);
    return rc;
}

void to_abi(const Tuning& t, uint32_t fill, uint32_t density, uint32_t scenes, float before, float after,
            nxm_tuning* out) {
    out->p2g_ctas_per_sm = t.p2g_ctas;
    out->g2p_ctas_per_sm = t.g2p_ctas;
    out->sort_ctas_per_sm = t.sort_ctas;
    out->grid_ctas_per_sm = t.grid_ctas;
    out->sort_batch = t.sort_batch;
    out->range_min_fill = fill;
    out->density = density;
    out->scenes = scenes;
    out->ms_before = before;
    out->ms_after = after;
}

}  // namespace

int nxm_state_autotune(nxm_state* s, uint32_t trial_steps, nxm_tuning* out) {
    if (!s) return NXM_E_INVALID;
    int rc = ensure_ready(s);
    if (rc) return rc;
    if (s->n == 0) return NXM_OK;
    static nxm_pipeline* pipe = nullptr;  // nxm_step takes a pipeline handle; it holds no state
    if (!pipe && (rc = nxm_pipeline_create(&pipe))) return rc;
    uint32_t density = 0, scenes = 0;
    bool known = false;
    NXM_TRY_RC(tune_key(s, &density, &scenes, &known));
    if (!known) {  // the counts come from a step
        NXM_TRY_RC(nxm_step(pipe, s, nullptr));
        NXM_TRY_RC(tune_key(s, &density, &scenes, &known));
    }
    const uint64_t key = ((uint64_t)density << 32) | scenes;
    if (trial_steps == 0) {  // apply the table's decision for this kind of state, if any
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tune_table.find(key);
        if (it != g_tune_table.end()) {
            apply_tuning(s, it->second.t, it->second.fill);
            if (out) to_abi(it->second.t, it->second.fill, density, scenes, it->second.ms_before, it->second.ms_after, out);
        } else if (out) {
            to_abi(s->tuning, s->range_min_fill, density, scenes, 0.f, 0.f, out);
        }
        return NXM_OK;
    }
    Tuning best = s->tuning;
    uint32_t best_fill = s->range_min_fill;
    float before = 0.f;
    NXM_TRY_RC(time_steps(pipe, s, trial_steps, &before));
    float best_ms = before;
    static const uint32_t kBatch[] = {2, 4, 8}, kSortCtas[] = {4, 8, 16}, kP2g[] = {2, 3}, kG2p[] = {3, 4},
                          kGrid[] = {4, 8, 16}, kFill[] = {16, 32, 64, 128, 256};
    struct Knob {
        uint32_t* field;  // inside `trial`
        const uint32_t* vals;
        int nvals;
    };
    Tuning trial = best;
    uint32_t trial_fill = best_fill;
    const Knob knobs[] = {{&trial.sort_batch, kBatch, 3}, {&trial.sort_ctas, kSortCtas, 3}, {&trial.p2g_ctas, kP2g, 2},
                          {&trial.g2p_ctas, kG2p, 2},     {&trial.grid_ctas, kGrid, 3},     {&trial_fill, kFill, 5}};
    for (const Knob& k : knobs) {
        trial = best;
        trial_fill = best_fill;
        const uint32_t keep = *k.field;
        for (int i = 0; i < k.nvals; ++i) {
            if (k.vals[i] == keep) continue;
            trial = best;
            trial_fill = best_fill;
            *k.field = k.vals[i];
            apply_tuning(s, trial, trial_fill);
            float ms = 0.f;
            NXM_TRY_RC(time_steps(pipe, s, trial_steps, &ms));
            if (ms < best_ms * 0.99f) {  // a clear win only
                best_ms = ms;
                best = trial;
                best_fill = trial_fill;
            }
        }
    }
    apply_tuning(s, best, best_fill);
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        g_tune_table[key] = TuneEntry{best, best_fill, before, best_ms};
    }
    if (out) to_abi(best, best_fill, density, scenes, before, best_ms, out);
    return NXM_OK;
}

int nxm_state_get_tuning(const nxm_state* s, nxm_tuning* out) {
    if (!s || !out) return NXM_E_INVALID;
    to_abi(s->tuning, s->range_min_fill, 0u, 0u, 0.f, 0.f, out);
    return NXM_OK;
}

int nxm_state_set_tuning(nxm_state* s, const nxm_tuning* t) {
    if (!s || !t) return NXM_E_INVALID;
    auto in = [](uint32_t v, std::initializer_list<uint32_t> ok) {
        for (uint32_t o : ok)
            if (v == o) return true;
        return false;
    };
    if (!in(t->p2g_ctas_per_sm, {1, 2, 3}) || !in(t->g2p_ctas_per_sm, {1, 2, 3, 4}) ||
        !in(t->sort_ctas_per_sm, {1, 2, 4, 8, 16}) || !in(t->grid_ctas_per_sm, {1, 2, 4, 8, 16}) ||
        !in(t->sort_batch, {2, 4, 8}) || t->range_min_fill == 0)
        return NXM_E_INVALID;
    Tuning x;
    x.p2g_ctas = t->p2g_ctas_per_sm;
    x.g2p_ctas = t->g2p_ctas_per_sm;
    x.sort_ctas = t->sort_ctas_per_sm;
    x.grid_ctas = t->grid_ctas_per_sm;
    x.sort_batch = t->sort_batch;
    apply_tuning(s, x, t->range_min_fill);
    return NXM_OK;
}

uint32_t nxm_tuning_table(nxm_tuning* out, uint32_t max_entries) {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    uint32_t i = 0;
    for (const auto& kv : g_tune_table) {
        if (out && i < max_entries)
            to_abi(kv.second.t, kv.second.fill, (uint32_t)(kv.first >> 32), (uint32_t)kv.first, kv.second.ms_before,
                   kv.second.ms_after, &out[i]);
        ++i;
    }
    return i;
}

int nxm_state_read_status_async(nxm_state* s, uint32_t* out, uint64_t* ticket) {
    if (!s || !out || !ticket) return NXM_E_INVALID;
    NXM_TRY(cudaMemcpyAsync(out, reinterpret_cast<const char*>(s->d_counters) + offsetof(Counters, status),
                            sizeof(uint32_t), cudaMemcpyDeviceToHost, s->stream));
    return nxm_state_fence(s, ticket);
}

int nxm_host_alloc(size_t bytes, void** out) {
    if (!out) return NXM_E_INVALID;
    *out = nullptr;
    const cudaError_t e = cudaMallocHost(out, std::max<size_t>(bytes, 1));
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        *out = nullptr;
        return e == cudaErrorMemoryAllocation ? NXM_E_OOM : NXM_E_CUDA;
    }
    return NXM_OK;
}

void nxm_host_free(void* p) {
    if (p) cudaFreeHost(p);
}

int nxm_state_status(nxm_state* s, uint32_t* bits, int clear) {
    if (!s || !bits) return NXM_E_INVALID;
    NXM_TRY(cudaMemcpyAsync(s->h_counters, s->d_counters, sizeof(Counters), cudaMemcpyDeviceToHost, s->stream));
    NXM_TRY(cudaStreamSynchronize(s->stream));
    *bits = s->h_counters->status;
    if (clear) {
        uint32_t z = 0;
        NXM_TRY(cudaMemcpyAsync(reinterpret_cast<char*>(s->d_counters) + offsetof(Counters, status), &z, 4,
                                cudaMemcpyHostToDevice, s->stream));
        NXM_TRY(cudaStreamSynchronize(s->stream));
    }
    return NXM_OK;
}

uint64_t nxm_state_kernel_launches(const nxm_state* s) { return s ? s->launches : 0; }

void* nxm_state_cuda_stream(const nxm_state* s) { return s ? reinterpret_cast<void*>(s->stream) : nullptr; }

// ---- readback ---------------------------------------------------------------

int nxm_read_positions(nxm_state* s, float* out) {
    if (!s) return NXM_E_INVALID;
    static const int off[3] = {0, 1, 2};
    return pack_read(s, s->kin, sizeof(PKin), off, 3, out);
}
int nxm_read_velocities(nxm_state* s, float* out) {
    if (!s) return NXM_E_INVALID;
    static const int off[3] = {4, 5, 6};
    return pack_read(s, s->kin, sizeof(PKin), off, 3, out);
}
int nxm_read_affine(nxm_state* s, float* out) {
    if (!s) return NXM_E_INVALID;
    static const int off[9] = {8, 9, 10, 12, 13, 14, 16, 17, 18};
    return pack_read(s, s->kin, sizeof(PKin), off, 9, out);
}
int nxm_read_vel_grad_det(nxm_state* s, float* out) {
    if (!s) return NXM_E_INVALID;
    static const int off[1] = {11};
    return pack_read(s, s->kin, sizeof(PKin), off, 1, out);
}
int nxm_read_mass(nxm_state* s, float* out) {
    if (!s) return NXM_E_INVALID;
    static const int off[1] = {3};
    return pack_read(s, s->kin, sizeof(PKin), off, 1, out);
}
int nxm_read_enabled(nxm_state* s, uint32_t* out) {
    if (!s || !out) return NXM_E_INVALID;
    static const int off[1] = {7};
    int rc = pack_read(s, s->kin, sizeof(PKin), off, 1, out);
    if (rc) return rc;
    for (uint32_t i = 0; i < s->n; ++i) out[i] = (out[i] & PFLAG_ENABLED) ? 1u : 0u;
    return NXM_OK;
}
int nxm_read_def_grad(nxm_state* s, float* out) {
    if (!s) return NXM_E_INVALID;
    static const int off[9] = {0, 1, 2, 4, 5, 6, 8, 9, 10};
    return pack_read(s, s->def, sizeof(PDef), off, 9, out);
}
int nxm_read_models(nxm_state* s, nxm_particle_model* out) {
    if (!s || !out) return NXM_E_INVALID;
    if (s->n == 0) return NXM_OK;
    std::vector<uint32_t> mid(s->n);
    static const int off_m[1] = {11};
    int rc = pack_read(s, s->def, sizeof(PDef), off_m, 1, mid.data());
    if (rc) return rc;
    std::vector<float> st(4 * (size_t)s->n);
    static const int off_s[4] = {0, 1, 2, 3};
    rc = pack_read(s, s->pstate, sizeof(float4), off_s, 4, st.data());
    if (rc) return rc;
    for (uint32_t i = 0; i < s->n; ++i) {
        if (mid[i] >= s->materials.size()) return NXM_E_INVALID;
        const Material& m = s->materials[mid[i]];
        out[i].tag = m.tag;
        const int ns = model_state_words(m.tag);
        for (int k = 0; k < MODEL_WORDS; ++k) out[i].data[k] = k < ns ? f_bits(st[4 * (size_t)i + k]) : f_bits(m.w[k]);
    }
    return NXM_OK;
}

// ---- grid inspection ----------------------------------------------------------

int nxm_grid_num_blocks(nxm_state* s, uint32_t* out) {
    if (!s || !out) return NXM_E_INVALID;
    NXM_TRY(cudaMemcpyAsync(s->h_counters, s->d_counters, sizeof(Counters), cudaMemcpyDeviceToHost, s->stream));
    NXM_TRY(cudaStreamSynchronize(s->stream));
    *out = s->h_counters->num_blocks;
    return NXM_OK;
}

int nxm_grid_sorted_len(nxm_state* s, uint32_t* out) {
    if (!s || !out) return NXM_E_INVALID;
    NXM_TRY(cudaMemcpyAsync(s->h_counters, s->d_counters, sizeof(Counters), cudaMemcpyDeviceToHost, s->stream));
    NXM_TRY(cudaStreamSynchronize(s->stream));
    *out = s->h_counters->sorted_len;
    return NXM_OK;
}

int nxm_grid_read_headers(nxm_state* s, int32_t* out, uint32_t max_blocks) {
    if (!s || !out) return NXM_E_INVALID;
    uint32_t nb = 0;
    int rc = nxm_grid_num_blocks(s, &nb);
    if (rc) return rc;
    nb = std::min(nb, max_blocks);
    if (nb == 0) return NXM_OK;
    std::vector<int4> v(nb);
    std::vector<uint32_t> f(nb), np(nb), nw(nb), cur((size_t)nb * NUM_BUCKETS), nbh((size_t)nb * NUM_NBH);
    NXM_TRY(cudaMemcpyAsync(v.data(), s->bvid, sizeof(int4) * nb, cudaMemcpyDeviceToHost, s->stream));
    NXM_TRY(cudaMemcpyAsync(f.data(), s->first, 4 * nb, cudaMemcpyDeviceToHost, s->stream));
    NXM_TRY(cudaMemcpyAsync(np.data(), s->nprim, 4 * nb, cudaMemcpyDeviceToHost, s->stream));
    NXM_TRY(cudaMemcpyAsync(nw.data(), s->nwx, 4 * nb, cudaMemcpyDeviceToHost, s->stream));
    NXM_TRY(cudaMemcpyAsync(cur.data(), s->cursors, 4 * cur.size(), cudaMemcpyDeviceToHost, s->stream));
    NXM_TRY(cudaMemcpyAsync(nbh.data(), s->nbh, 4 * nbh.size(), cudaMemcpyDeviceToHost, s->stream));
    NXM_TRY(cudaStreamSynchronize(s->stream));
    for (uint32_t b = 0; b < nb; ++b) {
        int32_t* o = out + 23 * (size_t)b;
        o[0] = v[b].x; o[1] = v[b].y; o[2] = v[b].z;
        o[3] = (int32_t)f[b]; o[4] = (int32_t)np[b]; o[5] = (int32_t)nw[b];
        for (int k = 0; k < NUM_BUCKETS; ++k) o[6 + k] = (int32_t)cur[(size_t)b * NUM_BUCKETS + k];
        for (int k = 0; k < NUM_NBH; ++k) o[16 + k] = (int32_t)nbh[(size_t)b * NUM_NBH + k];
    }
    return NXM_OK;
}

int nxm_grid_read_sorted_ids(nxm_state* s, uint32_t* out, uint32_t max_len) {
    if (!s || !out) return NXM_E_INVALID;
    uint32_t len = 0;
    int rc = nxm_grid_sorted_len(s, &len);
    if (rc) return rc;
    len = std::min(len, std::min(max_len, s->pcap * 8u));
    if (len == 0) return NXM_OK;
    NXM_TRY(cudaMemcpyAsync(out, s->sorted, 4 * (size_t)len, cudaMemcpyDeviceToHost, s->stream));
    std::vector<uint32_t> ids;
    if (s->sort_pid) {  // the sort listed storage slots: report particle ids
        ids.resize(s->n);
        NXM_TRY(cudaMemcpyAsync(ids.data(), s->sort_pid, 4 * (size_t)s->n, cudaMemcpyDeviceToHost, s->stream));
    }
    NXM_TRY(cudaStreamSynchronize(s->stream));
    if (s->sort_pid)
        for (uint32_t j = 0; j < len; ++j) out[j] = out[j] < s->n ? ids[out[j]] : out[j];
    return NXM_OK;
}

int nxm_grid_read_nodes(nxm_state* s, float* out, uint32_t max_blocks) {
    if (!s || !out) return NXM_E_INVALID;
    uint32_t nb = 0;
    int rc = nxm_grid_num_blocks(s, &nb);
    if (rc) return rc;
    nb = std::min(nb, max_blocks);
    if (nb == 0) return NXM_OK;
    NXM_TRY(cudaMemcpyAsync(out, s->nodes, sizeof(float4) * 64 * (size_t)nb, cudaMemcpyDeviceToHost, s->stream));
    NXM_TRY(cudaStreamSynchronize(s->stream));
    return NXM_OK;
}

}  // extern "C"
