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
// staged in shared memory in chunks of kP2gChunk: each staged record holds
// q = m v + C (x_0 - x_p) (x_0 = stencil node (0,0,0)), m, C dx and the
// three per-axis B-spline weight triples, so that the contribution to
// stencil node s is w_x[s.x] w_y[s.y] w_z[s.z] (q + (C dx) s, m).  The chunk
// is binned by associated cell (counting sort in shared memory); then each
// warp takes one cell at a time with lane l < 27 owning stencil offset s(l):
// the lanes read the cell's particles by broadcast and accumulate in
// registers, and one shared atomic per lane and component adds the cell's
// sum to the 6x6x6 node tile (the block plus the first two node layers of
// its +1 neighbours).  The tile goes to global memory with one float4
// atomic per non-empty node; nodes were zeroed by the sort.
constexpr int kP2gThreads = 256;
#ifndef NXM_P2G_CHUNK
#define NXM_P2G_CHUNK 512
#endif
#ifndef NXM_P2G_MIN_CTAS
#define NXM_P2G_MIN_CTAS 3
#endif
constexpr int kP2gChunk = NXM_P2G_CHUNK;  // particles staged per pass
constexpr int kP2gRec = 24;  // floats per staged particle
// record layout: [0..3] q.xyz, m | [4..12] (C dx) columns 0,1,2 | [13..15] w_x | [16..18] w_y | [19..21] w_z
constexpr size_t kP2gSmem = (size_t)kP2gChunk * kP2gRec * 4 + 216 * 16 + (64 + 68) * 4 + kP2gChunk * (2 + 2 + 1);

__global__ void __launch_bounds__(kP2gThreads, NXM_P2G_MIN_CTAS) k_p2g(DevPtrs P) {
    extern __shared__ float4 p2g_smem[];
    float* rec = reinterpret_cast<float*>(p2g_smem);
    float* tile = rec + kP2gChunk * kP2gRec;  // 216 x (x, y, z, m)
    int* cnt = reinterpret_cast<int*>(tile + 216 * 4);
    int* start = cnt + 64;  // 65 used
    uint16_t* perm = reinterpret_cast<uint16_t*>(start + 68);
    uint16_t* prank = perm + kP2gChunk;
    uint8_t* pcell = reinterpret_cast<uint8_t*>(prank + kP2gChunk);

    const float dx = P.params->dx;
    const float inv_dx = P.params->inv_dx;
    const uint32_t nb = P.counters->num_blocks;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    const int sx = (int)(lane % 3u), sy = (int)((lane / 3u) % 3u), sz = (int)(lane / 9u);
    for (uint32_t b = blockIdx.x; b < nb; b += gridDim.x) {
        const uint32_t first = P.first[b], np = P.nprim[b];
        if (np == 0) continue;  // neighbour-only block: receives its sums from other CTAs
        for (uint32_t t = tid; t < 216u * 4u; t += kP2gThreads) tile[t] = 0.f;
        if (tid < 64) cnt[tid] = 0;
        __syncthreads();
        const int4 vid = P.bvid[b];
        for (uint32_t base = 0; base < np; base += kP2gChunk) {
            const uint32_t m_chunk = min(np - base, (uint32_t)kP2gChunk);
            // 1. stage and bin
            for (uint32_t k = tid; k < m_chunk; k += kP2gThreads) {
                const uint32_t pid = P.sorted[first + base + k];
                const float4* kr = reinterpret_cast<const float4*>(&P.kin[pid]);
                const float4 xm = __ldg(kr), vf = __ldg(kr + 1);
                if (!(__float_as_uint(vf.w) & PFLAG_ENABLED)) {
                    pcell[k] = 255;
                    continue;
                }
                const float4 c0 = __ldg(kr + 2), c1 = __ldg(kr + 3), c2 = __ldg(kr + 4);
                const v3 pt = mk(xm.x, xm.y, xm.z);
                const float m = xm.w;
                const CellInfo ci = cell_info(dx, pt);
                const v3 r = mk((float)(vid.x * 4 + (int)ci.ax), (float)(vid.y * 4 + (int)ci.ay),
                                (float)(vid.z * 4 + (int)ci.az)) * dx - pt;
                const v3 wx = kernel_eval_all(-r.x * inv_dx);
                const v3 wy = kernel_eval_all(-r.y * inv_dx);
                const v3 wz = kernel_eval_all(-r.z * inv_dx);
                const m3 C = mkm(mk(c0.x, c0.y, c0.z), mk(c1.x, c1.y, c1.z), mk(c2.x, c2.y, c2.z));
                const v3 q = C * r + mk(vf.x, vf.y, vf.z) * m;
                float4* rr = reinterpret_cast<float4*>(rec + k * kP2gRec);
                rr[0] = make_float4(q.x, q.y, q.z, m);
                rr[1] = make_float4(C.c0.x * dx, C.c0.y * dx, C.c0.z * dx, C.c1.x * dx);
                rr[2] = make_float4(C.c1.y * dx, C.c1.z * dx, C.c2.x * dx, C.c2.y * dx);
                rr[3] = make_float4(C.c2.z * dx, wx.x, wx.y, wx.z);
                rr[4] = make_float4(wy.x, wy.y, wy.z, wz.x);
                rr[5] = make_float4(wz.y, wz.z, 0.f, 0.f);
                const uint32_t c = ci.ax + 4u * ci.ay + 16u * ci.az;
                pcell[k] = (uint8_t)c;
                prank[k] = (uint16_t)atomicAdd(&cnt[c], 1);
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
            for (uint32_t k = tid; k < m_chunk; k += kP2gThreads) {
                const uint32_t c = pcell[k];
                if (c != 255u) perm[start[c] + prank[k]] = (uint16_t)k;
            }
            __syncthreads();
            // 3. one warp per cell, lane = stencil offset
            for (uint32_t c = warp; c < 64u; c += kP2gThreads / 32) {
                const int s0 = start[c], s1 = start[c + 1];
                if (s0 == s1) continue;
                float ax = 0.f, ay = 0.f, az = 0.f, am = 0.f;
                for (int i = s0; i < s1; ++i) {
                    const float* r = rec + (uint32_t)perm[i] * kP2gRec;
                    const float4 qm = *reinterpret_cast<const float4*>(r);
                    const float4 c4a = *reinterpret_cast<const float4*>(r + 4);
                    const float4 c4b = *reinterpret_cast<const float4*>(r + 8);
                    const float c22 = r[12];
                    const float w = r[13 + sx] * r[16 + sy] * r[19 + sz];
                    const float fx = (float)sx, fy = (float)sy, fz = (float)sz;
                    const float vx = qm.x + c4a.x * fx + c4a.w * fy + c4b.z * fz;
                    const float vy = qm.y + c4a.y * fx + c4b.x * fy + c4b.w * fz;
                    const float vz = qm.z + c4a.z * fx + c4b.y * fy + c22 * fz;
                    ax += w * vx;
                    ay += w * vy;
                    az += w * vz;
                    am += w * qm.w;
                }
                if (lane < 27u) {
                    const uint32_t cx = c & 3u, cy = (c >> 2) & 3u, cz = c >> 4;
                    const uint32_t node = (cx + sx) + 6u * (cy + sy) + 36u * (cz + sz);
                    atomicAdd(&tile[node * 4 + 0], ax);
                    atomicAdd(&tile[node * 4 + 1], ay);
                    atomicAdd(&tile[node * 4 + 2], az);
                    atomicAdd(&tile[node * 4 + 3], am);
                }
            }
            __syncthreads();
            if (tid < 64) cnt[tid] = 0;
            __syncthreads();
        }
        for (uint32_t t = tid; t < 216u; t += kP2gThreads) {
            const float a = tile[4 * t], bb = tile[4 * t + 1], cc = tile[4 * t + 2], m = tile[4 * t + 3];
            if (a == 0.f && bb == 0.f && cc == 0.f && m == 0.f) continue;
            const uint32_t tx = t % 6u, ty = (t / 6u) % 6u, tz = t / 36u;
            const uint32_t ox = tx >= 4u, oy = ty >= 4u, oz = tz >= 4u;
            const uint32_t oct = ox * 4u + oy * 2u + oz;
            const uint32_t blk = oct == 0 ? b : P.nbh[b * NUM_NBH + oct - 1u];
            if (blk == NONE) {
                set_status_f(P.counters, STATUS_MISSING_BLOCK);
                continue;
            }
            const uint32_t node = blk * 64u + (tx - 4u * ox) + 4u * (ty - 4u * oy) + 16u * (tz - 4u * oz);
            atomicAdd(&P.nodes[node], make_float4(a, bb, cc, m));
        }
        __syncthreads();
    }
}

// rigid_impulses.rs:167-185: world centre of mass from the current pose.
__global__ void k_colliders_begin(DevPtrs P) {
    const uint32_t i = threadIdx.x;
    if (i >= P.params->ncol || i >= (uint32_t)MAX_COLLIDERS) return;
    DevCollider& c = P.colliders[i];
    quat q = quat{c.rot[0], c.rot[1], c.rot[2], c.rot[3]};
    v3 com = qrot(q, mk(c.local_com[0], c.local_com[1], c.local_com[2])) + mk(c.tra[0], c.tra[1], c.tra[2]);
    c.com[0] = com.x; c.com[1] = com.y; c.com[2] = com.z;
}

// dynamics/body.rs Velocity::integrate for one-way coupled bodies
// (rigid_impulses.rs:66-140 with zero impulse and zero inverse mass).
__global__ void k_colliders_end(DevPtrs P) {
    const uint32_t i = threadIdx.x;
    if (i >= P.params->ncol || i >= (uint32_t)MAX_COLLIDERS) return;
    const float dt = P.params->dt;
    DevCollider& c = P.colliders[i];
    quat q = quat{c.rot[0], c.rot[1], c.rot[2], c.rot[3]};
    v3 tra = mk(c.tra[0], c.tra[1], c.tra[2]);
    v3 init_com = qrot(q, mk(c.local_com[0], c.local_com[1], c.local_com[2])) + tra;
    v3 sa = mk(c.angvel[0], c.angvel[1], c.angvel[2]) * dt;
    float ang = length(sa);
    quat dq;
    if (ang == 0.f) {
        dq = quat{0.f, 0.f, 0.f, 1.f};
    } else {
        v3 ax = sa / ang;
        float sh = sinf(ang * 0.5f), ch = cosf(ang * 0.5f);
        dq = quat{ax.x * sh, ax.y * sh, ax.z * sh, ch};
    }
    v3 dl = mk(c.linvel[0], c.linvel[1], c.linvel[2]) * dt;
    v3 nt = (init_com + qrot(dq, tra - init_com)) + dl;
    quat nr;
    nr.w = dq.w * q.w - dq.x * q.x - dq.y * q.y - dq.z * q.z;
    nr.x = dq.w * q.x + dq.x * q.w + dq.y * q.z - dq.z * q.y;
    nr.y = dq.w * q.y - dq.x * q.z + dq.y * q.w + dq.z * q.x;
    nr.z = dq.w * q.z + dq.x * q.y - dq.y * q.x + dq.z * q.w;
    float rl = 1.0f / sqrtf(nr.x * nr.x + nr.y * nr.y + nr.z * nr.z + nr.w * nr.w);
    c.rot[0] = nr.x * rl; c.rot[1] = nr.y * rl; c.rot[2] = nr.z * rl; c.rot[3] = nr.w * rl;
    c.tra[0] = nt.x; c.tra[1] = nt.y; c.tra[2] = nt.z;
}

}  // namespace

void launch_p2g(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s) {
    cudaFuncSetAttribute(k_p2g, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kP2gSmem);
    k_p2g<<<c.sm_count * NXM_P2G_MIN_CTAS, kP2gThreads, kP2gSmem, s>>>(P);
}

void launch_colliders_begin(const DevPtrs& P, cudaStream_t s) { k_colliders_begin<<<1, 32, 0, s>>>(P); }
void launch_colliders_end(const DevPtrs& P, cudaStream_t s) { k_colliders_end<<<1, 32, 0, s>>>(P); }

}  // namespace fast
}  // namespace nxm
