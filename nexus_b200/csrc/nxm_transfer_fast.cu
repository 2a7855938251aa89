// Fast-path transfers: scatter-form P2G with a shared-memory node tile and
// one vector atomic flush per touched node, plus the grid update and the
// fused G2P + particle update (shared with the deterministic build through
// nxm_transfer.inc.cuh), and the collider pose kernels.
#define NXM_NS fast
#include "nxm_transfer.inc.cuh"

namespace nxm {
namespace fast {
namespace {

__device__ __forceinline__ void set_status_f(Counters* c, uint32_t bit) { atomicOr(&c->status, bit); }

// P2G (solver/p2g.rs:64-351 computes the same node sums in gather form).
// One CTA per active block: each thread scatters one primary particle's
// 27 weighted contributions w * (m v + C (x_i - x_p)) and w * m into a
// 6x6x6 node tile in shared memory (the block and the first two node layers
// of its +1 neighbours); the tile is then added to global memory with one
// float4 atomic per non-empty node.  Nodes were zeroed by the sort.
__global__ void __launch_bounds__(256) k_p2g(DevPtrs P) {
    __shared__ float tmx[216], tmy[216], tmz[216], tm[216];
    const float dx = P.params->dx;
    const float inv_dx = P.params->inv_dx;
    const uint32_t nb = P.counters->num_blocks;
    for (uint32_t b = blockIdx.x; b < nb; b += gridDim.x) {
        for (uint32_t t = threadIdx.x; t < 216u; t += blockDim.x) {
            tmx[t] = 0.f; tmy[t] = 0.f; tmz[t] = 0.f; tm[t] = 0.f;
        }
        __syncthreads();
        const int4 vid = P.bvid[b];
        const uint32_t first = P.first[b], np = P.nprim[b];
        for (uint32_t k = threadIdx.x; k < np; k += blockDim.x) {
            const uint32_t pid = P.sorted[first + k];
            const float4* kr = reinterpret_cast<const float4*>(&P.kin[pid]);
            const float4 xm = __ldg(kr), vf = __ldg(kr + 1), c0 = __ldg(kr + 2), c1 = __ldg(kr + 3), c2 = __ldg(kr + 4);
            if (!(__float_as_uint(vf.w) & PFLAG_ENABLED)) continue;
            const v3 pt = mk(xm.x, xm.y, xm.z);
            const float m = xm.w;
            const CellInfo ci = cell_info(dx, pt);
            // offset from the particle to stencil node (0,0,0)
            const v3 r = mk((float)(vid.x * 4 + (int)ci.ax), (float)(vid.y * 4 + (int)ci.ay),
                            (float)(vid.z * 4 + (int)ci.az)) * dx - pt;
            const v3 wx = kernel_eval_all(-r.x * inv_dx);
            const v3 wy = kernel_eval_all(-r.y * inv_dx);
            const v3 wz = kernel_eval_all(-r.z * inv_dx);
            const m3 C = mkm(mk(c0.x, c0.y, c0.z), mk(c1.x, c1.y, c1.z), mk(c2.x, c2.y, c2.z));
            const v3 q = C * r + mk(vf.x, vf.y, vf.z) * m;
            const v3 cx = C.c0 * dx, cy = C.c1 * dx, cz = C.c2 * dx;
            const uint32_t base = ci.ax + 6u * ci.ay + 36u * ci.az;
#pragma unroll
            for (int sz = 0; sz < 3; ++sz) {
                const float wzs = vget(wz, sz);
                const v3 qz = q + cz * (float)sz;
#pragma unroll
                for (int sy = 0; sy < 3; ++sy) {
                    const float wyz = vget(wy, sy) * wzs;
                    const v3 qy = qz + cy * (float)sy;
#pragma unroll
                    for (int sx = 0; sx < 3; ++sx) {
                        const float w = vget(wx, sx) * wyz;
                        const v3 val = qy + cx * (float)sx;
                        const uint32_t idx = base + (uint32_t)(sx + 6 * sy + 36 * sz);
                        atomicAdd(&tmx[idx], w * val.x);
                        atomicAdd(&tmy[idx], w * val.y);
                        atomicAdd(&tmz[idx], w * val.z);
                        atomicAdd(&tm[idx], w * m);
                    }
                }
            }
        }
        __syncthreads();
        for (uint32_t t = threadIdx.x; t < 216u; t += blockDim.x) {
            const float a = tmx[t], bb = tmy[t], cc = tmz[t], m = tm[t];
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
    k_p2g<<<c.sm_count * 4, 256, 0, s>>>(P);
}

void launch_colliders_begin(const DevPtrs& P, cudaStream_t s) { k_colliders_begin<<<1, 32, 0, s>>>(P); }
void launch_colliders_end(const DevPtrs& P, cudaStream_t s) { k_colliders_end<<<1, 32, 0, s>>>(P); }

}  // namespace fast
}  // namespace nxm
