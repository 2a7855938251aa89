// Fast-path transfers: scatter-form P2G with a shared-memory node tile and
// one vector atomic flush per touched node, plus the grid update and the
// fused G2P + particle update (shared with the deterministic build through
// nxm_transfer.inc.cuh), and the collider pose kernels.
#define NXM_NS fast
#define NXM_FAST true
#include "nxm_transfer.inc.cuh"

namespace nxm {
namespace fast {
namespace {

__device__ __forceinline__ void set_status_f(Counters* c, uint32_t bit) { atomicOr(&c->status, bit); }

// P2G (solver/p2g.rs:64-351 computes the same node sums in gather form).
//
// One CTA per active block (grid-stride).  The block's primary particles are
// staged in shared memory in chunks of kP2gChunk.  A staged record holds
//   q = m v + C (x_0 - x_p)  (x_0 = stencil node (0,0,0)) and m,
//   the three columns of C dx, each carrying one z weight w_z[k] alongside,
//   the nine products w_x[i] w_y[j],
// so the contribution to stencil node s is w_x[s.x] w_y[s.y] w_z[s.z]
// (q + (C dx) s, m).  The chunk is binned by associated cell (counting sort
// in shared memory).  Each warp then takes one cell at a time: lane l < 27
// owns the stencil column (s.x, s.y) = ((l mod 9) mod 3, (l mod 9) / 3) for
// particle group l / 9, so a pass reads three particles (three broadcast
// addresses per load) and each lane accumulates its column's three nodes.  A
// three-way shuffle exchange leaves lane l with the cell's full sum for node
// (s.x, s.y, l / 9), which it adds to the warp's private 6x6x6 node tile
// (the block plus the first two node layers of its +1 neighbours): the 27
// lanes own distinct nodes and no other warp writes that tile, so no atomics.
// At the end of the block the warp tiles are summed and each non-empty node
// goes to global memory with one float4 atomic; nodes were zeroed by the sort.
#ifndef NXM_P2G_WARPS
#define NXM_P2G_WARPS 8
#endif
#ifndef NXM_P2G_CHUNK
#define NXM_P2G_CHUNK 256
#endif
#ifndef NXM_P2G_MIN_CTAS
#define NXM_P2G_MIN_CTAS 3
#endif
constexpr int kP2gWarps = NXM_P2G_WARPS;
constexpr int kP2gThreads = 32 * kP2gWarps;
constexpr int kP2gChunk = NXM_P2G_CHUNK;  // particles staged per pass
constexpr int kP2gRec = 28;  // floats per staged particle
// record: [0..3] q.xyz, m | [4..7] (C dx).c0, w_z[0] | [8..11] (C dx).c1, w_z[1]
//       | [12..15] (C dx).c2, w_z[2] | [16 + i + 3 j] w_x[i] w_y[j] | [25..27] unused
constexpr size_t kP2gSmem = (size_t)kP2gWarps * 216 * 16 + (size_t)kP2gChunk * kP2gRec * 4 + (64 + 68) * 4 +
                            (size_t)kP2gChunk * (2 + 2 + 1);
// CPIC adds the warps' incompatible-field tiles and the 216 tile nodes' affinity bits
constexpr size_t kP2gSmemCpic = kP2gSmem + (size_t)kP2gWarps * 216 * 16 + 218 * 4 + 16;
static_assert(kP2gChunk <= 65536, "staged particle indices are 16-bit");

__device__ __forceinline__ float4 f4add(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }

// One staged particle's raw record (kin words 0..19, CPIC: its affinity
// bits) and a block header.
struct P2gRaw {
    float4 xm, vf, c0, c1, c2;
    float aff;
};
struct P2gHdr {
    uint32_t first, np;
};

template <bool kCpic>
__device__ __forceinline__ P2gRaw p2g_load_raw(const DevPtrs& P, uint32_t pid) {
    P2gRaw r;
    r.aff = 0.f;
    if (pid == NONE) {
        r.vf = make_float4(0.f, 0.f, 0.f, 0.f);  // flags 0: not staged
        return r;
    }
    const float4* kr = reinterpret_cast<const float4*>(&P.kin[pid]);
    r.xm = __ldg(kr);
    r.vf = __ldg(kr + 1);
    r.c0 = __ldg(kr + 2);
    r.c1 = __ldg(kr + 3);
    r.c2 = __ldg(kr + 4);
    // CPIC keeps particles in id order (slot = id): the affinity of this step's g2p_cdf
    if (kCpic) r.aff = __ldg(&P.pcdf[3u * pid + 1u].w);
    return r;
}

__device__ __forceinline__ P2gHdr p2g_load_hdr(const DevPtrs& P, uint32_t b, uint32_t nbp) {
    P2gHdr h{0u, 0u};
    if (b < nbp) {
        h.first = __ldcg(&P.first[b]);
        h.np = __ldcg(&P.nprim[b]);
    }
    return h;
}

// Work runs over the primary blocks only (ids [0, num_primary); the others
// hold no particles).  Loads run ahead of use: the headers of the blocks two
// grid strides ahead, the sorted id of the next chunk's particle right after
// staging, and its 80-byte record at the start of the cell phase, so their
// latency overlaps the current chunk's shared-memory work.
//
// CPIC (kCpic; solver/p2g.rs:258-310): a particle whose affinity bits are
// incompatible with a node's (aff_compatible) feeds that node's second,
// incompatible field instead: each lane keeps both sums for its three nodes,
// and the warps keep a second tile flushed into nodes_inc.
template <bool kCpic>
__global__ void __launch_bounds__(kP2gThreads, kCpic ? 2 : NXM_P2G_MIN_CTAS) k_p2g(DevPtrs P) {
    static_assert(kP2gChunk == kP2gThreads, "one staged particle per thread");
    static_assert(kP2gThreads >= 216, "one flushed tile node per thread");
    extern __shared__ float4 p2g_smem[];
    float4* tiles = p2g_smem;  // kP2gWarps x 216 nodes of (x, y, z, m)
    float4* tiles_inc = tiles + kP2gWarps * 216;  // CPIC only
    float* rec = reinterpret_cast<float*>(tiles + (kCpic ? 2 : 1) * kP2gWarps * 216);
    int* cnt = reinterpret_cast<int*>(rec + kP2gChunk * kP2gRec);
    int* start = cnt + 64;  // 65 used
    uint16_t* perm = reinterpret_cast<uint16_t*>(start + 68);
    uint16_t* prank = perm + kP2gChunk;
    uint8_t* pcell = reinterpret_cast<uint8_t*>(prank + kP2gChunk);
    uint32_t* node_aff = reinterpret_cast<uint32_t*>(pcell + ((kP2gChunk + 15) & ~15));  // CPIC: 216 tile nodes
    // CPIC: nonzero when a tile node of the current block carries an affinity
    // bit; otherwise every particle is compatible with every node and the
    // block runs the plain accumulation (no incompatible sums, no flush).
    // Two flags by block parity: the one of the next block is cleared while
    // the current one is in use (between two end-of-block barriers).
    volatile uint32_t* blk_aff_pair = node_aff + 216;
    uint32_t parity = 0u;

    const float dx = P.params->dx;
    const float inv_dx = P.params->inv_dx;
#ifndef NXM_P2G_POW2
#define NXM_P2G_POW2 1
#endif
    // a power-of-two cell width divides exactly by multiplying with its
    // reciprocal (the association must round as the reference's division)
    const uint32_t dxb = __float_as_uint(dx);
    const bool pow2 = NXM_P2G_POW2 && (dxb & 0x807FFFFFu) == 0u && (dxb >> 23) - 1u < 253u;
    const float rdx = __uint_as_float((254u << 23) - dxb);
    const uint32_t nbp = min(__ldcg(&P.counters->num_primary), __ldcg(&P.counters->num_blocks));
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    // cell-phase roles; lanes 27..31 idle (zero weight, never write)
    const bool worker = lane < 27u;
    const uint32_t grp = worker ? lane / 9u : 0u;
    const uint32_t sxy = worker ? lane % 9u : 0u;
    const float fx = (float)(sxy % 3u), fy = (float)(sxy / 3u);
    const uint32_t src1 = worker ? sxy + 9u * ((grp + 1u) % 3u) : lane;
    const uint32_t src2 = worker ? sxy + 9u * ((grp + 2u) % 3u) : lane;
    float4* tile = tiles + warp * 216u;
    float4* tile_inc = tiles_inc + warp * 216u;
    // flush role: tile node `tid` (tid < 216) of octant `foct`
    const uint32_t ftx = tid % 6u, fty = (tid / 6u) % 6u, ftz = tid / 36u;
    const uint32_t fox = ftx >= 4u, foy = fty >= 4u, foz = ftz >= 4u;
    const uint32_t foct = fox * 4u + foy * 2u + foz;
    const uint32_t fnode = (ftx - 4u * fox) + 4u * (fty - 4u * foy) + 16u * (ftz - 4u * foz);

    uint32_t b = blockIdx.x;
    if (b >= nbp) return;
    const uint32_t stride = gridDim.x;
    for (uint32_t t = tid; t < (kCpic ? 2u : 1u) * kP2gWarps * 216u; t += kP2gThreads)
        tiles[t] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (tid < 64) cnt[tid] = 0;
    if (kCpic && tid == 0) blk_aff_pair[0] = 0u;
    P2gHdr h = p2g_load_hdr(P, b, nbp);
    P2gHdr hn = p2g_load_hdr(P, b + stride, nbp);
    P2gHdr hnn = p2g_load_hdr(P, b + 2u * stride, nbp);
    P2gRaw raw = p2g_load_raw<kCpic>(P, tid < h.np ? __ldg(&P.sorted[h.first + tid]) : NONE);
    __syncthreads();
    for (;;) {
        int4 vid = P.bvid[b];
        {
            const int3 o = scene_base_of_block(*P.params, vid);  // scene-local block coordinates
            vid.x -= o.x; vid.y -= o.y; vid.z -= o.z;
        }
        const uint32_t fblk = (tid < 216u && foct != 0u) ? __ldg(&P.nbh[b * NUM_NBH + foct - 1u]) : b;
        volatile uint32_t* blk_aff = blk_aff_pair + parity;
        if (kCpic && tid == 0) blk_aff_pair[parity ^ 1u] = 0u;
        if (kCpic && tid < 216u) {  // read after the staging barrier below
            const uint32_t na = fblk == NONE ? 0u : __ldg(&P.ncdf[fblk * 64u + fnode].y);
            node_aff[tid] = na;
            if (na & 0x0000FFFFu) *blk_aff = 1u;
        }
        for (uint32_t base = 0; base < h.np; base += kP2gChunk) {
            const uint32_t m_chunk = min(h.np - base, (uint32_t)kP2gChunk);
            // 1. stage and bin this thread's particle (base + tid)
            if (tid < m_chunk) {
                const uint32_t k = tid;
                if (!(__float_as_uint(raw.vf.w) & PFLAG_ENABLED)) {
                    pcell[k] = 255;
                } else {
                    const v3 pt = mk(raw.xm.x, raw.xm.y, raw.xm.z);
                    const float m = raw.xm.w;
                    const CellInfo ci = pow2 ? cell_info_scaled(pt * rdx) : cell_info(dx, pt);
                    const v3 r = mk((float)(vid.x * 4 + (int)ci.ax), (float)(vid.y * 4 + (int)ci.ay),
                                    (float)(vid.z * 4 + (int)ci.az)) * dx - pt;
                    const v3 wx = kernel_eval_all(-r.x * inv_dx);
                    const v3 wy = kernel_eval_all(-r.y * inv_dx);
                    const v3 wz = kernel_eval_all(-r.z * inv_dx);
                    const m3 C = mkm(mk(raw.c0.x, raw.c0.y, raw.c0.z), mk(raw.c1.x, raw.c1.y, raw.c1.z),
                                     mk(raw.c2.x, raw.c2.y, raw.c2.z));
                    const v3 q = C * r + mk(raw.vf.x, raw.vf.y, raw.vf.z) * m;
                    float4* rr = reinterpret_cast<float4*>(rec + k * kP2gRec);
                    rr[0] = make_float4(q.x, q.y, q.z, m);
                    rr[1] = make_float4(C.c0.x * dx, C.c0.y * dx, C.c0.z * dx, wz.x);
                    rr[2] = make_float4(C.c1.x * dx, C.c1.y * dx, C.c1.z * dx, wz.y);
                    rr[3] = make_float4(C.c2.x * dx, C.c2.y * dx, C.c2.z * dx, wz.z);
                    rr[4] = make_float4(wx.x * wy.x, wx.y * wy.x, wx.z * wy.x, wx.x * wy.y);
                    rr[5] = make_float4(wx.y * wy.y, wx.z * wy.y, wx.x * wy.z, wx.y * wy.z);
                    rr[6] = make_float4(wx.z * wy.z, raw.aff, 0.f, 0.f);
                    const uint32_t c = ci.ax + 4u * ci.ay + 16u * ci.az;
                    pcell[k] = (uint8_t)c;
                    prank[k] = (uint16_t)atomicAdd(&cnt[c], 1);
                }
            }
            // sorted id of this thread's particle in the next chunk (this block or the next one)
            uint32_t pid_next = NONE;
            if (base + kP2gChunk < h.np) {
                if (base + kP2gChunk + tid < h.np) pid_next = __ldg(&P.sorted[h.first + base + kP2gChunk + tid]);
            } else if (tid < hn.np) {
                pid_next = __ldg(&P.sorted[hn.first + tid]);
            }
            __syncthreads();
            // 2. exclusive scan of the 64 cell counts
            if (warp == 0) {
                const int v0 = cnt[2 * lane], v1 = cnt[2 * lane + 1];
                int incl = v0 + v1;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
                    if ((int)lane >= o) incl += y;
                }
                const int excl = incl - v0 - v1;
                start[2 * lane] = excl;
                start[2 * lane + 1] = excl + v0;
                if (lane == 31) start[64] = incl;
            }
            __syncthreads();
            if (tid < m_chunk) {
                const uint32_t c = pcell[tid];
                if (c != 255u) perm[start[c] + prank[tid]] = (uint16_t)tid;
            }
            __syncthreads();
            if (tid < 64) cnt[tid] = 0;  // counts are consumed; ready for the next chunk
            raw = p2g_load_raw<kCpic>(P, pid_next);
            const bool split = kCpic && *blk_aff != 0u;
            // 3. one warp per cell, three particles per pass
            for (uint32_t c = warp; c < 64u; c += kP2gWarps) {
                const int s0 = start[c], s1 = start[c + 1];
                if (s0 == s1) continue;
                float4 a0 = make_float4(0.f, 0.f, 0.f, 0.f), a1 = a0, a2 = a0;  // s.z = 0, 1, 2
                float4 i0 = a0, i1 = a0, i2 = a0;  // CPIC: the incompatible sums
                const uint32_t cx = c & 3u, cy = (c >> 2) & 3u, cz = c >> 4;
                const uint32_t col = (cx + sxy % 3u) + 6u * (cy + sxy / 3u) + 36u * cz;  // this lane's s.z = 0 node
                uint32_t na0 = 0u, na1 = 0u, na2 = 0u;
                if (split && worker) {
                    na0 = node_aff[col];
                    na1 = node_aff[col + 36u];
                    na2 = node_aff[col + 72u];
                }
                for (int i = s0; i < s1; i += 3) {
                    const int j = i + (int)grp;
                    const bool valid = worker && j < s1;
                    const float* r = rec + (uint32_t)perm[valid ? j : s0] * kP2gRec;
                    const float4 qm = *reinterpret_cast<const float4*>(r);
                    const float4 k0 = *reinterpret_cast<const float4*>(r + 4);
                    const float4 k1 = *reinterpret_cast<const float4*>(r + 8);
                    const float4 k2 = *reinterpret_cast<const float4*>(r + 12);
                    const float wxy = valid ? r[16 + sxy] : 0.f;
                    float bx = qm.x + k0.x * fx + k1.x * fy;
                    float by = qm.y + k0.y * fx + k1.y * fy;
                    float bz = qm.z + k0.z * fx + k1.z * fy;
                    if (!split) {
                        float w = wxy * k0.w;
                        a0.x += w * bx; a0.y += w * by; a0.z += w * bz; a0.w += w * qm.w;
                        bx += k2.x; by += k2.y; bz += k2.z;
                        w = wxy * k1.w;
                        a1.x += w * bx; a1.y += w * by; a1.z += w * bz; a1.w += w * qm.w;
                        bx += k2.x; by += k2.y; bz += k2.z;
                        w = wxy * k2.w;
                        a2.x += w * bx; a2.y += w * by; a2.z += w * bz; a2.w += w * qm.w;
                    } else {
                        const uint32_t paff = __float_as_uint(r[25]);
                        const auto acc = [&](float4& a, float4& ai, uint32_t na, float w) {
                            const bool comp = aff_compatible(paff, na);
                            const float wc = comp ? w : 0.f, wi = comp ? 0.f : w;
                            a.x += wc * bx; a.y += wc * by; a.z += wc * bz; a.w += wc * qm.w;
                            ai.x += wi * bx; ai.y += wi * by; ai.z += wi * bz; ai.w += wi * qm.w;
                        };
                        acc(a0, i0, na0, wxy * k0.w);
                        bx += k2.x; by += k2.y; bz += k2.z;
                        acc(a1, i1, na1, wxy * k1.w);
                        bx += k2.x; by += k2.y; bz += k2.z;
                        acc(a2, i2, na2, wxy * k2.w);
                    }
                }
                // lane (sxy, g) collects node (sxy, s.z = g) from the three groups:
                // from group g+1 its s.z = g sum, which that lane holds as (its g + 2) mod 3,
                // from group g+2 likewise as (its g + 1) mod 3.
                const auto exchange = [&](float4 x0, float4 x1, float4 x2) {
                    const float4 own = grp == 0u ? x0 : (grp == 1u ? x1 : x2);
                    const float4 out1 = grp == 0u ? x2 : (grp == 1u ? x0 : x1);
                    const float4 out2 = grp == 0u ? x1 : (grp == 1u ? x2 : x0);
                    float4 t;
                    t.x = own.x + __shfl_sync(0xFFFFFFFFu, out1.x, src1) + __shfl_sync(0xFFFFFFFFu, out2.x, src2);
                    t.y = own.y + __shfl_sync(0xFFFFFFFFu, out1.y, src1) + __shfl_sync(0xFFFFFFFFu, out2.y, src2);
                    t.z = own.z + __shfl_sync(0xFFFFFFFFu, out1.z, src1) + __shfl_sync(0xFFFFFFFFu, out2.z, src2);
                    t.w = own.w + __shfl_sync(0xFFFFFFFFu, out1.w, src1) + __shfl_sync(0xFFFFFFFFu, out2.w, src2);
                    return t;
                };
                const float4 t = exchange(a0, a1, a2);
                const uint32_t node = col + 36u * grp;
                if (worker) tile[node] = f4add(tile[node], t);
                if (split) {
                    const float4 ti = exchange(i0, i1, i2);
                    if (worker) tile_inc[node] = f4add(tile_inc[node], ti);
                }
            }
            __syncthreads();
        }
        // 4. sum the warp tiles (clearing them) and flush the block's nodes
        const int nfields = kCpic && *blk_aff != 0u ? 2 : 1;
        if (tid < 216u) {
            for (int f = 0; f < nfields; ++f) {
                float4* tt = f ? tiles_inc : tiles;
                float4 sum = tt[tid];
                tt[tid] = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int w = 1; w < kP2gWarps; ++w) {
                    sum = f4add(sum, tt[w * 216 + tid]);
                    tt[w * 216 + tid] = make_float4(0.f, 0.f, 0.f, 0.f);
                }
                if (sum.x != 0.f || sum.y != 0.f || sum.z != 0.f || sum.w != 0.f) {
                    if (fblk == NONE) set_status_f(P.counters, STATUS_MISSING_BLOCK);
                    else atomicAdd(&(f ? P.nodes_inc : P.nodes)[fblk * 64u + fnode], sum);
                }
            }
        }
        __syncthreads();
        parity ^= 1u;
        b += stride;
        if (b >= nbp) break;
        h = hn;
        hn = hnn;
        hnn = p2g_load_hdr(P, b + 2u * stride, nbp);
    }
}

}  // namespace

void launch_p2g(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s) {
    cudaFuncSetAttribute(k_p2g<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kP2gSmem);
    k_p2g<false><<<c.sm_count * (int)min(c.t.p2g_ctas, (uint32_t)NXM_P2G_MIN_CTAS), kP2gThreads, kP2gSmem, s>>>(P);
}

void launch_p2g_cpic(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s) {
    cudaFuncSetAttribute(k_p2g<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kP2gSmemCpic);
    k_p2g<true><<<c.sm_count * 2, kP2gThreads, kP2gSmemCpic, s>>>(P);
}


}  // namespace fast
}  // namespace nxm
