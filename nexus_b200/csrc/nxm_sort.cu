// Block activation and particle sort (src_mpm/grid/grid.rs:26-191,
// src_mpm_shaders/grid/sort.rs:104-491, src_mpm_shaders/grid/grid.rs:447-578).
//
// Same results as the reference: the set of active blocks (every particle's
// 2x2x2 block neighbourhood), the per-block slab buckets (4 primary z-slabs,
// 6 extra buckets), the +1 neighbour header ids and the sorted id list.
// Header order and the order inside a bucket come from atomics, as in the
// reference; the canonical pass (deterministic mode) orders every bucket by
// ascending particle id.  The extras (a particle listed again in each +1
// neighbour block its stencil reaches) are only built when asked for: the
// gather-form P2G reads them, the scatter-form P2G does not.
//
// B200 specifics: every particle pass is a persistent grid-stride loop that
// keeps whole warps together, so that __match_any_sync can merge the atomics
// of lanes that hit the same block (or the same block bucket): one hash probe
// or one atomicAdd per distinct key per warp instead of one per particle.
// The block key of each particle is cached in `pcode` (8 bytes) by the
// previous step's G2P, so activation does not re-read the 80-byte particle
// records.  Counters, headers and the hash live in L2.
#include "nxm_device.cuh"
#include "nxm_kernels.h"

// k_count<false> / k_finalize<false> skip the extras loop by design.
#pragma nv_diag_suppress 128

namespace nxm {
namespace {

__device__ __forceinline__ void set_status(Counters* c, uint32_t bit) { atomicOr(&c->status, bit); }

__device__ __forceinline__ void assoc_shift(int i, int& dx, int& dy, int& dz) {
    // grid.rs:175-212 blocks_associated_to_block: z fastest.
    dx = (i >> 2) & 1;
    dy = (i >> 1) & 1;
    dz = i & 1;
}

// Insert `key` (block kx,ky,kz); allocates a header on first insertion.
// Primary blocks take ids [0, num_primary); neighbour-pass blocks take ids
// base + [0, num_extra) with base = num_primary.
__device__ void hash_insert(const DevPtrs& P, uint32_t key, int kx, int ky, int kz, bool primary, uint32_t base,
                            uint32_t hash_mask, uint32_t block_cap) {
    uint32_t slot = hash_key(key) & hash_mask;
    for (uint32_t it = 0; it <= hash_mask; ++it) {
        uint32_t cur = __ldcg(&P.hkey[slot]);
        if (cur == key) return;
        if (cur == NONE) {
            uint32_t old = atomicCAS(&P.hkey[slot], NONE, key);
            if (old == NONE) {
                uint32_t id = primary ? atomicAdd(&P.counters->num_primary, 1u)
                                      : base + atomicAdd(&P.counters->num_extra, 1u);
                if (id >= block_cap) {
                    set_status(P.counters, STATUS_BLOCK_CAPACITY);
                    P.hval[slot] = NONE;
                    return;
                }
                P.bvid[id] = make_int4(kx, ky, kz, (int)key);
                P.hval[slot] = id;
                return;
            }
            if (old == key) return;
        }
        slot = (slot + 1) & hash_mask;
    }
    set_status(P.counters, STATUS_HASH_FULL);
}

__device__ __forceinline__ uint32_t hash_find(const DevPtrs& P, uint32_t key, uint32_t hash_mask) {
    uint32_t slot = hash_key(key) & hash_mask;
    for (uint32_t it = 0; it <= hash_mask; ++it) {
        uint32_t cur = __ldg(&P.hkey[slot]);
        if (cur == key) return __ldg(&P.hval[slot]);
        if (cur == NONE) return NONE;
        slot = (slot + 1) & hash_mask;
    }
    return NONE;
}

// Warp-aggregated atomicAdd: lanes with equal `key` (NONE = no-op) share one
// atomic; each gets base + its rank among the equal lanes (lane order).
__device__ __forceinline__ uint32_t warp_agg_add(uint32_t key, uint32_t* addr) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t peers = __match_any_sync(0xFFFFFFFFu, key);
    uint32_t leader = __ffs(peers) - 1;
    uint32_t rank = __popc(peers & ((1u << lane) - 1u));
    uint32_t base = 0;
    if (key != NONE && lane == leader) base = atomicAdd(addr, (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    return base + rank;
}

// Warp-aggregated atomicAdd without a result (fire-and-forget).
__device__ __forceinline__ void warp_agg_red(uint32_t key, uint32_t* addr) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, key);
    if (key != NONE && lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(addr, (uint32_t)__popc(peers));
}

// The contiguous particle range [lo, hi) of this warp (a multiple of 32 long):
// with particles stored in block order, a warp's consecutive passes mostly see
// the same block, which lets the passes below skip repeated hash work.
__device__ __forceinline__ void warp_range(uint32_t n, uint32_t& lo, uint32_t& hi) {
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t per_warp = ((n + nwarps - 1) / nwarps + 31u) & ~31u;
    lo = min(warp * per_warp, n);
    hi = min(lo + per_warp, n);
}

// kSortBatch (a template parameter of the particle passes): passes of 32
// particles whose loads a warp issues together (2, 4 or 8; tuned per state).

__device__ __forceinline__ bool spills(uint32_t ax, uint32_t ay, uint32_t az, int sx, int sy, int sz) {
    // sort.rs:320-329, EXTRA_PARTICLE_MIN_SHIFT = 2
    return (sx == 0 || ax >= 2) && (sy == 0 || ay >= 2) && (sz == 0 || az >= 2);
}
__device__ __forceinline__ uint32_t extra_bucket(uint32_t az, int sz) {
    // sort.rs:56-62
    int local = (int)az - sz * 4;
    if (local < -2) local = -2;
    return NUM_PRIMARY_BUCKETS + (uint32_t)(local + 2);
}

// ---------------------------------------------------------------------------

// Clears the hash and the step counters; the last CTA also refreshes the
// colliders' world centres of mass from their poses (rigid_impulses.rs:167-185),
// which the grid update reads.
__global__ void k_sort_reset(DevPtrs P, uint32_t hash_cap) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < hash_cap; i += gridDim.x * blockDim.x)
        P.hkey[i] = NONE;
    if (P.colliders && blockIdx.x == gridDim.x - 1) {
        const Params& prm = *P.params;
        const uint32_t ncol = prm.scene_blocks ? prm.ncol : min(prm.ncol, (uint32_t)MAX_COLLIDERS);
        for (uint32_t i = threadIdx.x; i < ncol; i += blockDim.x) {
            DevCollider& c = P.colliders[i];
            const quat q = quat{c.rot[0], c.rot[1], c.rot[2], c.rot[3]};
            const v3 com = qrot(q, mk(c.local_com[0], c.local_com[1], c.local_com[2])) + mk(c.tra[0], c.tra[1], c.tra[2]);
            c.com[0] = com.x; c.com[1] = com.y; c.com[2] = com.z;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        P.counters->num_primary = 0;
        P.counters->num_extra = 0;
        P.counters->num_blocks = 0;
        P.counters->sorted_len = 0;
        P.counters->unsorted = 0;
        P.counters->rigid_len = 0;
    }
}

// sort.rs:104-121 gpu_touch_primary_blocks.  Block keys come from the cache
// written by the previous step (or from the positions after an upload).
// Each warp walks a contiguous range of particles, so consecutive passes
// mostly see the block they inserted last: a pass whose lanes all carry the
// key inserted by the previous pass skips the hash entirely.
template <int kSortBatch>
__global__ void __launch_bounds__(256) k_touch_primary(DevPtrs P) {
    const uint32_t n = P.params->n;
    const float dx = P.params->dx;
    const uint32_t hmask = P.params->hash_capacity - 1;
    const uint32_t bcap = P.params->block_capacity;
    const bool cached = P.counters->codes_valid != 0;
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t lo, hi;
    warp_range(n, lo, hi);
    uint32_t known = NONE;  // a key this warp has already inserted
    for (uint32_t base = lo; base < hi; base += 32u * kSortBatch) {
        uint32_t keys[kSortBatch];
#pragma unroll
        for (int j = 0; j < kSortBatch; ++j) {
            const uint32_t p = base + 32u * j + lane;
            uint32_t key = NONE;
            if (p < hi) {
                if (cached) {
                    key = __ldg(&P.pcode[p].x);
                } else {
                    float4 xm = __ldg(reinterpret_cast<const float4*>(&P.kin[p]));
                    CellInfo ci = cell_info(dx, mk(xm.x, xm.y, xm.z));
                    int3 o = make_int3(0, 0, 0);
                    if (P.params->scene_blocks) o = scene_base_of(*P.params, P.pscene[P.pid_in ? P.pid_in[p] : p]);
                    key = pack_key(ci.bx + o.x, ci.by + o.y, ci.bz + o.z);
                    P.pcode[p] = make_uint2(key, ci.ax | (ci.ay << 2) | (ci.az << 4));
                }
            }
            keys[j] = key;
        }
#pragma unroll
        for (int j = 0; j < kSortBatch; ++j) {
            const uint32_t b32 = base + 32u * j;
            if (b32 >= hi) break;
            const bool active = b32 + lane < hi;
            const uint32_t key = keys[j];
            const uint32_t need = (active && key != known) ? key : NONE;
            if (!__all_sync(0xFFFFFFFFu, need == NONE)) {
                const uint32_t peers = __match_any_sync(0xFFFFFFFFu, need);
                if (need != NONE && lane == (uint32_t)(__ffs(peers) - 1))
                    hash_insert(P, key, key_x(key), key_y(key), key_z(key), true, 0, hmask, bcap);
            }
            // the last active lane's key is now in the table
            known = __shfl_sync(0xFFFFFFFFu, key, min(31u, hi - 1u - b32));
        }
    }
}

// sort.rs:133-163 gpu_touch_neighbor_blocks: one thread per (base block, neighbour).
__global__ void __launch_bounds__(256) k_touch_nbh(DevPtrs P) {
    const uint32_t hmask = P.params->hash_capacity - 1;
    const uint32_t bcap = P.params->block_capacity;
    const uint32_t nprim = min(__ldcg(&P.counters->num_primary), bcap);
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nprim * 7u; t += gridDim.x * blockDim.x) {
        const uint32_t b = t / 7u;
        const int i = (int)(t % 7u) + 1;
        const int4 v = P.bvid[b];
        int sx, sy, sz;
        assoc_shift(i, sx, sy, sz);
        const int kx = v.x + sx, ky = v.y + sy, kz = v.z + sz;
        hash_insert(P, pack_key(kx, ky, kz), kx, ky, kz, false, nprim, hmask, bcap);
    }
}

// sort.rs:261-279 gpu_update_nbh_block_ids, plus zeroing of the block's
// bucket counters and P2G accumulation nodes.  One thread per node.
__global__ void __launch_bounds__(256) k_block_prep(DevPtrs P) {
    const uint32_t hmask = P.params->hash_capacity - 1;
    const uint32_t bcap = P.params->block_capacity;
    const uint32_t nprim = min(__ldcg(&P.counters->num_primary), bcap);
    const uint32_t total = min(nprim + __ldcg(&P.counters->num_extra), bcap);
    if (blockIdx.x == 0 && threadIdx.x == 0) P.counters->num_blocks = total;
    const uint32_t nthreads = total * 64u;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nthreads; t += gridDim.x * blockDim.x) {
        const uint32_t b = t >> 6, k = t & 63u;
        if (P.nodes) P.nodes[t] = make_float4(0.f, 0.f, 0.f, 0.f);
        // the scatter P2G of CPIC accumulates the incompatible field too
        if (P.nodes_inc && P.params->use_cpic) P.nodes_inc[t] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (k < NUM_NBH) {
            int4 v = P.bvid[b];
            int sx, sy, sz;
            assoc_shift((int)k + 1, sx, sy, sz);
            P.nbh[b * NUM_NBH + k] = hash_find(P, pack_key(v.x + sx, v.y + sy, v.z + sz), hmask);
        } else if (k < NUM_NBH + NUM_BUCKETS) {
            P.cursors[b * NUM_BUCKETS + (k - NUM_NBH)] = 0;
        } else if (k == 63u && P.rp_count) {
            P.rp_count[b] = 0;
        }
    }
}

// sort.rs:287-349 gpu_update_block_particle_count.
template <bool kExtras, int kSortBatch>
__global__ void __launch_bounds__(256) k_count(DevPtrs P) {
    const uint32_t n = P.params->n;
    const uint32_t hmask = P.params->hash_capacity - 1;
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t lo, hi;
    warp_range(n, lo, hi);
    uint32_t known_key = NONE, known_h0 = NONE;  // the last key this warp looked up
    for (uint32_t base = lo; base < hi; base += 32u * kSortBatch) {
        uint2 codes[kSortBatch];
#pragma unroll
        for (int j = 0; j < kSortBatch; ++j) {
            const uint32_t p = base + 32u * j + lane;
            codes[j] = p < hi ? P.pcode[p] : make_uint2(NONE, 0u);
        }
#pragma unroll
        for (int j = 0; j < kSortBatch; ++j) {
            const uint32_t b32 = base + 32u * j;
            if (b32 >= hi) break;
            const uint32_t p = b32 + lane;
            const bool active = p < hi;
            const uint2 code = codes[j];
            const uint32_t key = active ? code.x : NONE;
            uint32_t h0;
            if (__all_sync(0xFFFFFFFFu, !active || key == known_key)) {
                h0 = active ? known_h0 : NONE;
            } else {  // one probe per distinct block key in the warp
                const uint32_t peers = __match_any_sync(0xFFFFFFFFu, key);
                const uint32_t leader = __ffs(peers) - 1;
                uint32_t h = NONE;
                if (active && lane == leader) h = hash_find(P, key, hmask);
                h0 = __shfl_sync(0xFFFFFFFFu, h, leader);
            }
            const uint32_t last = min(31u, hi - 1u - b32);
            known_key = __shfl_sync(0xFFFFFFFFu, key, last);
            known_h0 = __shfl_sync(0xFFFFFFFFu, h0, last);
            if (active) {
                P.phdr[p] = h0;
                if (h0 == NONE) set_status(P.counters, STATUS_MISSING_BLOCK);
            }
            const uint32_t ax = code.y & 3u, ay = (code.y >> 2) & 3u, az = (code.y >> 4) & 3u;
            const uint32_t bkey = (h0 != NONE) ? h0 * 16u + az : NONE;
            warp_agg_red(bkey, bkey != NONE ? &P.cursors[h0 * NUM_BUCKETS + az] : nullptr);
            if (!kExtras) continue;
            for (int i = 1; i < 8; ++i) {
                int sx, sy, sz;
                assoc_shift(i, sx, sy, sz);
                uint32_t hn = NONE, e = 0;
                if (h0 != NONE && spills(ax, ay, az, sx, sy, sz)) {
                    hn = P.nbh[h0 * NUM_NBH + (i - 1)];
                    if (hn == NONE) set_status(P.counters, STATUS_MISSING_BLOCK);
                    e = extra_bucket(az, sz);
                }
                const uint32_t k2 = (hn != NONE) ? hn * 16u + e : NONE;
                warp_agg_red(k2, k2 != NONE ? &P.cursors[hn * NUM_BUCKETS + e] : nullptr);
            }
        }
    }
}

// prefix sum (src_rbd/utils/prefix_sum.rs) over the block totals, then
// sort.rs:382-420 gpu_copy_scan_values_to_first_particles, as a two-pass
// tiled scan: pass 1 gives each block its offset inside a tile of kScanTile
// blocks and each tile its total; pass 2 adds the tile's offset (the sum of
// the tile totals before it) and turns the bucket counts into cursors.
constexpr uint32_t kScanThreads = 256;
constexpr uint32_t kScanPer = kScanTile / kScanThreads;  // blocks per thread

// Exclusive CTA-wide scan of one value per thread; returns the CTA total in *total.
__device__ __forceinline__ uint32_t cta_exclusive_scan(uint32_t v, uint32_t* warp_tot, uint32_t* total) {
    const uint32_t lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= (uint32_t)o) incl += y;
    }
    if (lane == 31) warp_tot[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        const uint32_t nw = blockDim.x >> 5;
        uint32_t w = lane < nw ? warp_tot[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
            if (lane >= (uint32_t)o) wi += y;
        }
        if (lane < nw) warp_tot[lane] = wi - w;
        if (lane == 31) warp_tot[32] = wi;
    }
    __syncthreads();
    const uint32_t out = warp_tot[wid] + incl - v;
    *total = warp_tot[32];
    __syncthreads();
    return out;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(DevPtrs P) {
    __shared__ uint32_t warp_tot[33];
    const uint32_t total = P.counters->num_blocks;
    const uint32_t ntiles = (total + kScanTile - 1) / kScanTile;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const uint32_t b0 = tile * kScanTile + threadIdx.x * kScanPer;
        uint32_t bt[kScanPer];
        uint32_t t = 0;
#pragma unroll
        for (uint32_t j = 0; j < kScanPer; ++j) {
            const uint32_t b = b0 + j;
            uint32_t s = 0;
            if (b < total) {
#pragma unroll
                for (int k = 0; k < NUM_BUCKETS; ++k) s += P.cursors[b * NUM_BUCKETS + k];
            }
            bt[j] = s;
            t += s;
        }
        uint32_t tile_total;
        uint32_t run = cta_exclusive_scan(t, warp_tot, &tile_total);
#pragma unroll
        for (uint32_t j = 0; j < kScanPer; ++j) {
            const uint32_t b = b0 + j;
            if (b < total) P.scan_tmp[b] = run;
            run += bt[j];
        }
        if (threadIdx.x == 0) P.tile_sums[tile] = tile_total;
    }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_apply(DevPtrs P) {
    __shared__ uint32_t warp_tot[33];
    const uint32_t total = P.counters->num_blocks;
    const uint32_t ntiles = (total + kScanTile - 1) / kScanTile;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        uint32_t part = 0;
        for (uint32_t i = threadIdx.x; i < tile; i += kScanThreads) part += P.tile_sums[i];
        uint32_t offset;
        cta_exclusive_scan(part, warp_tot, &offset);
        const uint32_t b0 = tile * kScanTile + threadIdx.x * kScanPer;
        // all loads first: the stores below may alias them as far as the compiler knows
        uint32_t cnt[kScanPer][NUM_BUCKETS], rel[kScanPer];
#pragma unroll
        for (uint32_t j = 0; j < kScanPer; ++j) {
            const uint32_t b = b0 + j;
            rel[j] = b < total ? P.scan_tmp[b] : 0u;
#pragma unroll
            for (int k = 0; k < NUM_BUCKETS; ++k) cnt[j][k] = b < total ? P.cursors[b * NUM_BUCKETS + k] : 0u;
        }
#pragma unroll
        for (uint32_t j = 0; j < kScanPer; ++j) {
            const uint32_t b = b0 + j;
            if (b >= total) break;
            const uint32_t first = offset + rel[j];
            uint32_t running = first;
            P.first[b] = first;
#pragma unroll
            for (int k = 0; k < NUM_BUCKETS; ++k) {
                if (k == NUM_PRIMARY_BUCKETS) P.nprim[b] = running - first;
                P.cursors[b * NUM_BUCKETS + k] = running;
                running += cnt[j][k];
            }
            P.nwx[b] = running - first;
            // the runs of kRangeChunk sorted positions that start inside this block
            if (P.chunk_blk)
                for (uint32_t c = (first + kRangeChunk - 1u) / kRangeChunk; c * kRangeChunk < running && c < P.chunk_cap; ++c)
                    P.chunk_blk[c] = b;
            if (b == total - 1) {
                P.counters->sorted_len = running;
                if (running > P.params->sorted_capacity) set_status(P.counters, STATUS_SORT_CAPACITY);
            }
        }
    }
}

// sort.rs:430-491 gpu_finalize_particles_sort.
template <bool kExtras, int kSortBatch>
__global__ void __launch_bounds__(256) k_finalize(DevPtrs P) {
    const uint32_t n = P.params->n;
    const uint32_t scap = P.params->sorted_capacity;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt_mask = (1u << lane) - 1u;
    uint32_t lo, hi;
    warp_range(n, lo, hi);
    for (uint32_t base = lo; base < hi; base += 32u * kSortBatch) {
        uint32_t h0[kSortBatch], code[kSortBatch];
#pragma unroll
        for (int j = 0; j < kSortBatch; ++j) {
            const uint32_t p = base + 32u * j + lane;
            h0[j] = p < hi ? P.phdr[p] : NONE;
            code[j] = p < hi ? P.pcode[p].y : 0u;
        }
        // the bucket atomics of all passes in flight together, then the scatter
        uint32_t key[kSortBatch], leader[kSortBatch], rank[kSortBatch], got[kSortBatch];
#pragma unroll
        for (int j = 0; j < kSortBatch; ++j) {
            const uint32_t az = (code[j] >> 4) & 3u;
            key[j] = (h0[j] != NONE) ? h0[j] * 16u + az : NONE;
            const uint32_t peers = __match_any_sync(0xFFFFFFFFu, key[j]);
            leader[j] = __ffs(peers) - 1;
            rank[j] = __popc(peers & lt_mask);
            got[j] = 0u;
            if (key[j] != NONE && lane == leader[j])
                got[j] = atomicAdd(&P.cursors[h0[j] * NUM_BUCKETS + az], (uint32_t)__popc(peers));
        }
#pragma unroll
        for (int j = 0; j < kSortBatch; ++j) {
            const uint32_t p = base + 32u * j + lane;
            const uint32_t slot = __shfl_sync(0xFFFFFFFFu, got[j], leader[j]) + rank[j];
            if (key[j] != NONE && slot < scap) P.sorted[slot] = p;
            if (!kExtras) continue;
            const uint32_t ax = code[j] & 3u, ay = (code[j] >> 2) & 3u, az = (code[j] >> 4) & 3u;
            for (int i = 1; i < 8; ++i) {
                int sx, sy, sz;
                assoc_shift(i, sx, sy, sz);
                uint32_t hn = NONE, e = 0;
                if (h0[j] != NONE && spills(ax, ay, az, sx, sy, sz)) {
                    hn = P.nbh[h0[j] * NUM_NBH + (i - 1)];
                    e = extra_bucket(az, sz);
                }
                const uint32_t k2 = (hn != NONE) ? hn * 16u + e : NONE;
                const uint32_t s2 = warp_agg_add(k2, k2 != NONE ? &P.cursors[hn * NUM_BUCKETS + e] : nullptr);
                if (k2 != NONE && s2 < scap) P.sorted[s2] = p;
            }
        }
    }
}

// Canonical order: every (block, bucket) segment sorted by ascending id.
// Rank sort in shared memory (particle ids are distinct inside a block).
constexpr uint32_t kSegMax = 4096;
__global__ void __launch_bounds__(256) k_sort_segments(DevPtrs P) {
    __shared__ uint32_t buf[kSegMax];
    const uint32_t total = P.counters->num_blocks;
    for (uint32_t b = blockIdx.x; b < total; b += gridDim.x) {
        uint32_t start = P.first[b];
        for (int k = 0; k < NUM_BUCKETS; ++k) {
            const uint32_t end = P.cursors[b * NUM_BUCKETS + k];
            const uint32_t len = end - start;
            if (len > 1 && len <= kSegMax) {
                for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) buf[i] = P.sorted[start + i];
                __syncthreads();
                for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) {
                    const uint32_t v = buf[i];
                    uint32_t rank = 0;
                    for (uint32_t j = 0; j < len; ++j) rank += buf[j] < v ? 1u : 0u;
                    P.sorted[start + rank] = v;
                }
                __syncthreads();
            } else if (len > kSegMax && threadIdx.x == 0) {
                set_status(P.counters, STATUS_SORT_CAPACITY);
            }
            start = end;
        }
    }
}

inline int grid_for(int sm_count, int per_sm) { return sm_count * per_sm; }


// ---------------------------------------------------------------------------
// Primary-only sort of plain float4 positions (no per-particle scratch: the
// key is recomputed from the position in each pass and the primary block is
// found again through the hash).  Used by the allocation-free entry point.

__device__ __forceinline__ uint32_t key_of(const float4* pos, uint32_t p, float dx, uint32_t* assoc) {
    const float4 x = __ldg(&pos[p]);
    const CellInfo ci = cell_info(dx, mk(x.x, x.y, x.z));
    *assoc = ci.ax | (ci.ay << 2) | (ci.az << 4);
    return pack_key(ci.bx, ci.by, ci.bz);
}

__global__ void __launch_bounds__(256) k_touch_primary_pos(DevPtrs P, const float4* __restrict__ pos) {
    const uint32_t n = P.params->n;
    const float dx = P.params->dx;
    const uint32_t hmask = P.params->hash_capacity - 1;
    const uint32_t bcap = P.params->block_capacity;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t base = warp * 32u; base < n; base += nwarps * 32u) {
        const uint32_t p = base + lane;
        uint32_t assoc = 0, key = NONE;
        if (p < n) key = key_of(pos, p, dx, &assoc);
        uint32_t peers = __match_any_sync(0xFFFFFFFFu, key);
        if (p < n && lane == (uint32_t)(__ffs(peers) - 1))
            hash_insert(P, key, key_x(key), key_y(key), key_z(key), true, 0, hmask, bcap);
    }
}

template <bool kScatter>
__global__ void __launch_bounds__(256) k_bucket_pos(DevPtrs P, const float4* __restrict__ pos) {
    const uint32_t n = P.params->n;
    const float dx = P.params->dx;
    const uint32_t hmask = P.params->hash_capacity - 1;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t base = warp * 32u; base < n; base += nwarps * 32u) {
        const uint32_t p = base + lane;
        uint32_t h0 = NONE, assoc = 0;
        if (p < n) {
            h0 = hash_find(P, key_of(pos, p, dx, &assoc), hmask);
            if (h0 == NONE) set_status(P.counters, STATUS_MISSING_BLOCK);
        }
        const uint32_t az = (assoc >> 4) & 3u;
        const uint32_t key = (h0 != NONE) ? h0 * 16u + az : NONE;
        const uint32_t slot = warp_agg_add(key, key != NONE ? &P.cursors[h0 * NUM_BUCKETS + az] : nullptr);
        if (kScatter && key != NONE && slot < P.params->sorted_capacity) P.sorted[slot] = p;
    }
}

}  // namespace

int sort_launches(bool canonical) { return canonical ? 9 : 8; }

void launch_sort_positions(const DevPtrs& P, const LaunchCfg& c, const float4* pos, cudaStream_t s) {
    const int g = grid_for(c.sm_count, 8);
    int reset_grid = (int)((c.hash_capacity + 255u) / 256u);
    if (reset_grid > g) reset_grid = g;
    if (reset_grid < 1) reset_grid = 1;
    k_sort_reset<<<reset_grid, 256, 0, s>>>(P, c.hash_capacity);
    k_touch_primary_pos<<<g, 256, 0, s>>>(P, pos);
    k_touch_nbh<<<g, 256, 0, s>>>(P);
    k_block_prep<<<g, 256, 0, s>>>(P);
    k_bucket_pos<false><<<g, 256, 0, s>>>(P, pos);
    k_scan_tiles<<<c.sm_count, kScanThreads, 0, s>>>(P);
    k_scan_apply<<<c.sm_count, kScanThreads, 0, s>>>(P);
    k_bucket_pos<true><<<g, 256, 0, s>>>(P, pos);
}


// ---------------------------------------------------------------------------
// CPIC rigid particles (src_mpm/grid/grid.rs:95-121, sort.rs:165-249, 493-667).
// ---------------------------------------------------------------------------

namespace {

// Block (global key coordinates: in batched mode offset by the scene of the
// sample's collider, as the particles' keys are) and associated cell of rigid
// particle i.
__device__ __forceinline__ CellInfo rigid_cell(const DevPtrs& P, uint32_t i, float dx) {
    const float4 w = P.rp_world[i];
    CellInfo ci = cell_info(dx, mk(w.x, w.y, w.z));
    if (P.params->scene_blocks) {
        const uint32_t sid = P.colliders[__float_as_uint(w.w) >> kRigidTriBits].scene;
        const int3 o = scene_base_of(*P.params, sid);
        ci.bx += o.x;
        ci.by += o.y;
        ci.bz += o.z;
    }
    return ci;
}

// sort.rs:200-249 gpu_mark_rigid_particles_needing_block: a rigid particle
// needs its own block when that block is missing while one of its +1
// neighbours exists (without it the particle could not be listed there).
// Runs on the hash as the particle passes left it, before any insertion.
__global__ void __launch_bounds__(256) k_rigid_mark(DevPtrs P) {
    const uint32_t hmask = P.params->hash_capacity - 1;
    const float dx = P.params->dx;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.nrp; i += gridDim.x * blockDim.x) {
        const CellInfo ci = rigid_cell(P, i, dx);
        int k = 0;
        for (; k < 8; ++k) {
            int sx, sy, sz;
            assoc_shift(k, sx, sy, sz);
            if (hash_find(P, pack_key(ci.bx + sx, ci.by + sy, ci.bz + sz), hmask) != NONE) break;
        }
        P.rp_need[i] = (k > 0 && k < 8) ? 1u : 0u;
    }
}

// sort.rs:165-198 gpu_touch_rigid_particle_blocks: the marked particles'
// blocks join the neighbour-pass blocks (ids after the primaries).
__global__ void __launch_bounds__(256) k_rigid_touch(DevPtrs P) {
    const uint32_t hmask = P.params->hash_capacity - 1;
    const uint32_t bcap = P.params->block_capacity;
    const uint32_t nprim = min(__ldcg(&P.counters->num_primary), bcap);
    const float dx = P.params->dx;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.nrp; i += gridDim.x * blockDim.x) {
        if (!P.rp_need[i]) continue;
        const CellInfo ci = rigid_cell(P, i, dx);
        hash_insert(P, pack_key(ci.bx, ci.by, ci.bz), ci.bx, ci.by, ci.bz, false, nprim, hmask, bcap);
    }
}

// The blocks a rigid particle is listed in: its own block (NONE if missing:
// the particle is skipped) and each existing +1 neighbour its 3-cell range
// reaches (sort.rs:509-553).  Returns how many; out[0] is the own block.
__device__ __forceinline__ int rigid_blocks(const DevPtrs& P, uint32_t i, float dx, uint32_t hmask, uint32_t out[8]) {
    const CellInfo ci = rigid_cell(P, i, dx);
    const uint32_t h0 = hash_find(P, pack_key(ci.bx, ci.by, ci.bz), hmask);
    if (h0 == NONE) return 0;
    int n = 0;
    out[n++] = h0;
    for (int k = 1; k < 8; ++k) {
        int sx, sy, sz;
        assoc_shift(k, sx, sy, sz);
        if (!spills(ci.ax, ci.ay, ci.az, sx, sy, sz)) continue;
        const uint32_t hb = P.nbh[h0 * NUM_NBH + k - 1];
        if (hb != NONE) out[n++] = hb;
    }
    return n;
}

// sort.rs:493-556 gpu_update_block_rigid_particle_count.
__global__ void __launch_bounds__(256) k_rigid_count(DevPtrs P) {
    const uint32_t hmask = P.params->hash_capacity - 1;
    const float dx = P.params->dx;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.nrp; i += gridDim.x * blockDim.x) {
        uint32_t hb[8];
        const int n = rigid_blocks(P, i, dx, hmask, hb);
        for (int k = 0; k < n; ++k) atomicAdd(&P.rp_count[hb[k]], 1u);
    }
}

// Each block with rigid entries takes a contiguous range of the list (the
// reference lays the ranges out by a prefix sum, sort.rs:558-600; p2g_cdf
// reads one block's range, so the order of the ranges is free): one atomic
// per warp on the list length, a warp scan for the lanes' offsets.  The
// count becomes the placement cursor.
__global__ void __launch_bounds__(256) k_rigid_alloc(DevPtrs P) {
    const uint32_t nb = __ldcg(&P.counters->num_blocks);
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < nb; base += stride) {
        const uint32_t b = base + lane;
        const uint32_t cnt = b < nb ? P.rp_count[b] : 0u;
        uint32_t incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
            if (lane >= (uint32_t)o) incl += v;
        }
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        uint32_t start = 0;
        if (lane == 31u && total) start = atomicAdd(&P.counters->rigid_len, total);
        start = __shfl_sync(0xFFFFFFFFu, start, 31);
        if (b < nb) {
            P.rp_first[b] = start + incl - cnt;
            P.rp_count[b] = 0;
        }
    }
}

// sort.rs:602-667 gpu_finalize_rigid_particles_sort: the same block set as
// the count pass, so every claimed slot stays inside its block's range.
__global__ void __launch_bounds__(256) k_rigid_finalize(DevPtrs P) {
    const uint32_t hmask = P.params->hash_capacity - 1;
    const float dx = P.params->dx;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.nrp; i += gridDim.x * blockDim.x) {
        uint32_t hb[8];
        const int n = rigid_blocks(P, i, dx, hmask, hb);
        for (int k = 0; k < n; ++k) {
            const uint32_t slot = atomicAdd(&P.rp_count[hb[k]], 1u);
            P.rp_sorted[P.rp_first[hb[k]] + slot] = i;
        }
    }
}

}  // namespace

namespace fast {

void launch_sort(const DevPtrs& P, const LaunchCfg& c, bool with_extras, bool canonical, cudaStream_t s,
                 bool rigid) {
    const int g = grid_for(c.sm_count, (int)c.t.sort_ctas);
    int reset_grid = (int)((c.hash_capacity + 255u) / 256u);
    if (reset_grid > g) reset_grid = g;
    if (reset_grid < 1) reset_grid = 1;
    k_sort_reset<<<reset_grid, 256, 0, s>>>(P, c.hash_capacity);
    switch (c.t.sort_batch) {
    case 2: k_touch_primary<2><<<g, 256, 0, s>>>(P); break;
    case 8: k_touch_primary<8><<<g, 256, 0, s>>>(P); break;
    default: k_touch_primary<4><<<g, 256, 0, s>>>(P); break;
    }
    k_touch_nbh<<<g, 256, 0, s>>>(P);
    if (rigid) {
        k_rigid_mark<<<g, 256, 0, s>>>(P);
        k_rigid_touch<<<g, 256, 0, s>>>(P);
    }
    k_block_prep<<<g, 256, 0, s>>>(P);
    switch ((with_extras ? 16 : 0) + c.t.sort_batch) {
    case 2: k_count<false, 2><<<g, 256, 0, s>>>(P); break;
    case 8: k_count<false, 8><<<g, 256, 0, s>>>(P); break;
    case 18: k_count<true, 2><<<g, 256, 0, s>>>(P); break;
    case 20: k_count<true, 4><<<g, 256, 0, s>>>(P); break;
    case 24: k_count<true, 8><<<g, 256, 0, s>>>(P); break;
    default: k_count<false, 4><<<g, 256, 0, s>>>(P); break;
    }
    k_scan_tiles<<<c.sm_count, kScanThreads, 0, s>>>(P);
    k_scan_apply<<<c.sm_count, kScanThreads, 0, s>>>(P);
    switch ((with_extras ? 16 : 0) + c.t.sort_batch) {
    case 2: k_finalize<false, 2><<<g, 256, 0, s>>>(P); break;
    case 8: k_finalize<false, 8><<<g, 256, 0, s>>>(P); break;
    case 18: k_finalize<true, 2><<<g, 256, 0, s>>>(P); break;
    case 20: k_finalize<true, 4><<<g, 256, 0, s>>>(P); break;
    case 24: k_finalize<true, 8><<<g, 256, 0, s>>>(P); break;
    default: k_finalize<false, 4><<<g, 256, 0, s>>>(P); break;
    }
    if (canonical) k_sort_segments<<<grid_for(c.sm_count, 4), 256, 0, s>>>(P);
    if (rigid) {
        k_rigid_count<<<g, 256, 0, s>>>(P);
        k_rigid_alloc<<<g, 256, 0, s>>>(P);
        k_rigid_finalize<<<g, 256, 0, s>>>(P);
    }
}

}  // namespace fast
}  // namespace nxm
