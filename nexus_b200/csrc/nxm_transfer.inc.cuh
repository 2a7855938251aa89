// Grid update and G2P + particle update kernels, included twice: by
// nxm_transfer_fast.cu (multiply-adds may fuse) and by nxm_transfer_det.cu
// (built with --fmad=false, every multiply and add rounded separately in the
// reference's order).  NXM_NS names the namespace of the instantiation.
#include "nxm_device.cuh"
#include "nxm_kernels.h"

#ifndef NXM_NS
#error "define NXM_NS before including nxm_transfer.inc.cuh"
#endif
#ifndef NXM_FAST
#error "define NXM_FAST (true: fast build, false: reference operation order)"
#endif
#ifndef NXM_CPIC
#define NXM_CPIC 0  // 1: also build the CPIC branches (deterministic-build kernels only)
#endif

namespace nxm {
namespace NXM_NS {
namespace {

__device__ __forceinline__ void set_status(Counters* c, uint32_t bit) { atomicOr(&c->status, bit); }

__device__ __forceinline__ v3 col_vel_at(const DevCollider& c, v3 p) {
    // dynamics/body.rs:239-250 velocity_at_point
    v3 lin = mk(c.linvel[0], c.linvel[1], c.linvel[2]);
    v3 ang = mk(c.angvel[0], c.angvel[1], c.angvel[2]);
    v3 com = mk(c.com[0], c.com[1], c.com[2]);
    return lin + cross(ang, p - com);
}

struct Collision {
    v3 normal;
    float distance;
    uint32_t closest;
};

// Whether analytic collider c (ball, cuboid, capsule) can touch a node of a
// block whose 64 nodes lie within rb of `centre` (rb = 1.5 sqrt(3) dx about
// the block's middle): the exact distance at the centre, then the bound
// distance(node) >= distance(centre) - rb.  A contributing node is inside the
// shape or has its projection within cap on every axis (so within sqrt(3)
// cap): the collider is kept when the centre is inside or the shape lies
// within rb + sqrt(3) cap of it.  The reach carries a relative and an
// absolute margin above the rounding of the per-node queries it stands for.
__device__ __forceinline__ bool analytic_near_block(const DevCollider& c, float cap, float rb, v3 centre) {
    const quat q = quat{c.rot[0], c.rot[1], c.rot[2], c.rot[3]};
    const v3 local = qrot(qconj(q), centre - mk(c.tra[0], c.tra[1], c.tra[2]));
    Proj pr;
    if (c.type == SHAPE_BALL) pr = ball_project_local(c.a[0], local);
    else if (c.type == SHAPE_CUBOID) pr = cuboid_project_local(mk(c.a[0], c.a[1], c.a[2]), local);
    else if (c.type == SHAPE_CAPSULE)
        pr = capsule_project_local(mk(c.a[0], c.a[1], c.a[2]), mk(c.b[0], c.b[1], c.b[2]), c.b[3], local);
    else return true;
    if (pr.inside) return true;
    const v3 d = pr.point - local;
    const float reach = (rb + 1.75f * cap) * 1.001f + 1.0e-5f;
    return !(dot(d, d) > reach * reach);  // a NaN keeps the collider
}

// Whether trimesh collider c can have a triangle within cap of a node of the
// block: the box of its BVH root within rb + cap of the centre (a node's
// query descends only into boxes within cap of the node).  Only the root is
// tested: one lane's deeper query for the whole block costs the warp about
// as much as the 32 per-node queries it would save.
__device__ __forceinline__ bool mesh_near_block(const DevPtrs& P, const DevCollider& c, float cap, float rb,
                                                v3 centre) {
    if (c.bvh_count == 0u) return false;
    const quat ci = qconj(quat{c.rot[0], c.rot[1], c.rot[2], c.rot[3]});
    const v3 local = qrot(ci, centre) + (-qrot(ci, mk(c.tra[0], c.tra[1], c.tra[2])));
    return !(aabb_distance(P.bvh[c.bvh_first], local) > (rb + cap) * 1.001f + 1.0e-5f);
}

// Bit i: collider i (< 32) may touch a node of block `vid` (scene-local
// block coordinates).  Every lane of the warp calls it for the same block;
// lane i tests collider i.  Trimeshes are left out when `skip_meshes`.
__device__ __forceinline__ uint32_t colliders_near_block(const DevPtrs& P, const DevCollider* cols, uint32_t ncol,
                                                        float dx, int4 vid, bool skip_meshes) {
    const uint32_t lane = threadIdx.x & 31u;
    const v3 centre = mk((float)vid.x * 4.0f + 1.5f, (float)vid.y * 4.0f + 1.5f, (float)vid.z * 4.0f + 1.5f) * dx;
    const float cap = dx * 1.5f, rb = 2.6f * dx;
    bool near = false;
    if (lane < ncol) {
        const DevCollider& c = cols[lane];
        near = c.type == SHAPE_TRIMESH ? !skip_meshes && mesh_near_block(P, c, cap, rb, centre)
                                       : analytic_near_block(c, cap, rb, centre);
    }
    return __ballot_sync(0xFFFFFFFFu, near);
}

// `near` (bit i for collider i < 32, from colliders_near_block) leaves out
// the colliders that cannot reach this node: their projections would find
// no point within cap and no inside.
__device__ __forceinline__ Collision collide(const DevPtrs& P, const DevCollider* cols, uint32_t ncol, float dx,
                                             v3 point, uint32_t near) {
    const float cap = dx * 1.5f;
    Collision col;
    col.normal = splat(0.f);
    col.distance = MAX_FLT;
    col.closest = 0;
    for (uint32_t i = 0; i < ncol; ++i) {
        if (i < 32u && !(near & (1u << i))) {
            // next candidate: skip the run of unset bits at once
            const uint32_t rest = near & ~((2u << i) - 1u);
            if (rest == 0u) i = 31u;
            else i = (uint32_t)__ffs(rest) - 2u;
            continue;
        }
        const DevCollider& c = cols[i];
        quat q = quat{c.rot[0], c.rot[1], c.rot[2], c.rot[3]};
        v3 tra = mk(c.tra[0], c.tra[1], c.tra[2]);
        // fast build: an unrotated collider (the usual box walls) skips the
        // two rotations (the deterministic build keeps them: they turn -0 into +0)
        const bool ident = NXM_FAST && q.x == 0.f && q.y == 0.f && q.z == 0.f && q.w == 1.f;
        Proj pr;
        if (ident && c.type != SHAPE_TRIMESH) {
            const v3 local = point - tra;
            if (c.type == SHAPE_BALL) pr = ball_project_local(c.a[0], local);
            else if (c.type == SHAPE_CUBOID) pr = cuboid_project_local(mk(c.a[0], c.a[1], c.a[2]), local);
            else if (c.type == SHAPE_CAPSULE)
                pr = capsule_project_local(mk(c.a[0], c.a[1], c.a[2]), mk(c.b[0], c.b[1], c.b[2]), c.b[3], local);
            else { pr.point = local; pr.inside = false; }
            pr.point = pr.point + tra;
        } else if (c.type == SHAPE_TRIMESH) {
            // pose.inverse() * point, as the inverse isometry applies it
            const quat ci = qconj(q);
            const v3 local = qrot(ci, point) + (-qrot(ci, tra));
            if (!trimesh_project_local(P.tris, P.bvh, c.bvh_first, c.bvh_count, local, cap, pr)) continue;
        } else {
            v3 local = qrot(qconj(q), point - tra);
            if (c.type == SHAPE_BALL) pr = ball_project_local(c.a[0], local);
            else if (c.type == SHAPE_CUBOID) pr = cuboid_project_local(mk(c.a[0], c.a[1], c.a[2]), local);
            else if (c.type == SHAPE_CAPSULE)
                pr = capsule_project_local(mk(c.a[0], c.a[1], c.a[2]), mk(c.b[0], c.b[1], c.b[2]), c.b[3], local);
            else { pr.point = local; pr.inside = false; }
        }
        if (!(ident && c.type != SHAPE_TRIMESH)) pr.point = qrot(q, pr.point) + tra;
        v3 dpt = pr.point - point;
        v3 ad = vabs(dpt);
        bool within = ad.x <= cap && ad.y <= cap && ad.z <= cap;
        if (pr.inside || within) {
            float sign = pr.inside ? -1.0f : 1.0f;
            float distance = length(dpt);
            v3 normal = dpt / (distance * -sign);
            float sd = sign * distance;
            if (sd < col.distance) {
                col.distance = sd;
                col.normal = normal;
                col.closest = i;
            }
        }
    }
    return col;
}

// grid_update.rs:21-88 + grid_update_collide.rs:102-183, one thread per node.
__global__ void __launch_bounds__(256) k_grid_update(DevPtrs P) {
    __shared__ DevCollider scol[MAX_COLLIDERS];
    const Params prm = *P.params;
    // batched scenes: each block sees only its scene's colliders (global memory)
    const bool scenes = prm.scene_blocks != 0;
    const uint32_t ncol = prm.use_cpic ? 0u : (scenes ? prm.ncol : min(prm.ncol, (uint32_t)MAX_COLLIDERS));
    if (!scenes)
        for (uint32_t i = threadIdx.x; i < ncol * (sizeof(DevCollider) / 4); i += blockDim.x)
            reinterpret_cast<uint32_t*>(scol)[i] = reinterpret_cast<const uint32_t*>(P.colliders)[i];
    __syncthreads();
    const float dx = prm.dx, dt = prm.dt;
    const v3 g = mk(prm.gravity[0], prm.gravity[1], prm.gravity[2]);
    const float lim = dx / dt;
    const uint32_t total = P.counters->num_blocks * 64u;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        float4 nd = P.nodes[t];
        const float mass = nd.w;
        const float inv_mass = mass > 0.f ? 1.0f / mass : 0.0f;
        v3 v = (mk(nd.x, nd.y, nd.z) + g * (mass * dt)) * inv_mass;
        v = vclamp(v, -lim, lim);
        if (ncol > 0) {
            const uint32_t b = t >> 6, k = t & 63u;
            int4 vid = P.bvid[b];
            const DevCollider* cols = scol;
            uint32_t nc = ncol;
            if (scenes) {
                const uint32_t sid = scene_of_block(prm, vid);
                const uint2 r = sid != NONE ? P.scene_cols[sid] : make_uint2(0u, 0u);
                cols = P.colliders + r.x;
                nc = r.y;
                const int3 o = scene_base_of_block(prm, vid);  // scene-local node position
                vid.x -= o.x; vid.y -= o.y; vid.z -= o.z;
            }
            v3 cell_pt = mk((float)(vid.x * 4 + (int)(k & 3u)), (float)(vid.y * 4 + (int)((k >> 2) & 3u)),
                            (float)(vid.z * 4 + (int)(k >> 4))) * dx;
            // the warp's 32 nodes share one block: its colliders in reach, one lane each
            const uint32_t near = colliders_near_block(P, cols, nc, dx, vid, false);
            Collision c = collide(P, cols, nc, dx, cell_pt, near);
            if (c.distance != MAX_FLT) {
                const DevCollider& cc = cols[c.closest];
                v3 bv = col_vel_at(cc, cell_pt);
                v3 delta = v - bv;
                float nv = dot(delta, c.normal);
                const float margin = dx;
                if (c.distance <= margin) {
                    v = bv + bc_project(cc.bc_type, cc.bc_friction, delta, c.normal);
                } else if (-nv * dt > c.distance - margin) {
                    v3 excess = c.normal * (nv + (c.distance - margin) / dt);
                    v = v - excess;
                }
            }
        }
        P.nodes[t] = make_float4(v.x, v.y, v.z, mass);
#if NXM_CPIC
        if (prm.use_cpic) {  // grid_update.rs:55-66: the incompatible field gets the same update
            const float4 ni = P.nodes_inc[t];
            const float mi = ni.w;
            const float inv_mi = mi > 0.f ? 1.0f / mi : 0.0f;
            v3 vi = (mk(ni.x, ni.y, ni.z) + g * (mi * dt)) * inv_mi;
            vi = vclamp(vi, -lim, lim);
            P.nodes_inc[t] = make_float4(vi.x, vi.y, vi.z, mi);
        }
#endif
    }
}

// CPIC context of one block for G2P: the incompatible velocities and node
// distance fields of its 6x6x6 halo, and the colliders it sees.
struct CpicCtx {
    const float4* halo_inc;
    const uint2* halo_cdf;  // affinity bits, closest collider
    const DevCollider* cols;
    uint32_t ncols;
};

// Velocity of shared-halo node t (t = x + 6 y + 36 z, x, y, z in [0, 6)) of
// block b: node (x mod 4, ...) of the block itself or of one of its +1
// neighbours; zero where that neighbour is not active.
__device__ __forceinline__ float4 halo_node(const DevPtrs& P, uint32_t b, uint32_t t) {
    const uint32_t tx = t % 6u, ty = (t / 6u) % 6u, tz = t / 36u;
    const uint32_t ox = tx >= 4u, oy = ty >= 4u, oz = tz >= 4u;
    const uint32_t oct = ox * 4u + oy * 2u + oz;
    const uint32_t blk = oct == 0 ? b : P.nbh[b * NUM_NBH + oct - 1u];
    if (blk == NONE) return make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 nd = P.nodes[blk * 64u + (tx - 4u * ox) + 4u * (ty - 4u * oy) + 16u * (tz - 4u * oz)];
    return make_float4(nd.x, nd.y, nd.z, 0.f);
}

#ifndef NXM_G2P_THREADS
#define NXM_G2P_THREADS 256
#endif
constexpr uint32_t kG2pThreads = NXM_G2P_THREADS;  // threads per G2P CTA

// g2p.rs:150-270 (non-CPIC) fused with particle_update.rs:60-201 for one
// particle: gathers velocity and velocity gradient from the 6x6x6 halo of its
// block (shared memory), then advects, updates F and the model, and writes the
// particle (read from slot `src`, xm / vf = its first two kin words) to slot
// `dst` of the output records, together with the block key of its new position.
// kCpicBlock: the CPIC branches (a block whose halo carries affinity bits);
// the plain instantiation serves every other block without their registers.
template <bool kCpicBlock>
__device__ __forceinline__ void g2p_particle(const DevPtrs& P, const Params& prm, const float4* __restrict__ halo,
                                             uint32_t src, uint32_t dst, float4 xm, float4 vf, int3 key_off,
                                             const CpicCtx& cx, volatile float* stash) {
    const float dx = prm.dx, dt = prm.dt;
    const float inv_d = 4.0f / (dx * dx);
    float4* kr = reinterpret_cast<float4*>(&P.kin_out[dst]);
    uint32_t flags = __float_as_uint(vf.w);
    const v3 pt = mk(xm.x, xm.y, xm.z);
    float mass = xm.w;
    // the deformation record, loaded ahead of the gather
    const float4* dr = reinterpret_cast<const float4*>(&P.def[src]);
    const float4 d0 = dr[0], d1 = dr[1], d2 = dr[2];

#if NXM_CPIC
    // particle Cdf (normal, signed distance, affinity) from this step's g2p_cdf pass
    const bool cpic = kCpicBlock;
    float4 crec0 = make_float4(0.f, 0.f, 0.f, 0.f), crec1 = crec0;
    float bfric = 1.0f;
    if (cpic) {
        crec0 = P.pcdf[3u * src];
        crec1 = P.pcdf[3u * src + 1u];
        bfric = P.pcdf[3u * src + 2u].x;
    }
    const uint32_t paff = __float_as_uint(crec1.w);
    const v3 pnormal = mk(crec0.x, crec0.y, crec0.z);
    v3 rigid_vel = splat(0.f);
#else
    (void)cx;
#endif
    // ---- G2P (g2p.rs:150-270)
    v3 velocity = splat(0.f);
    m3 grad = mzero();
    float vgd = 0.f;
#if NXM_CPIC
    // a particle with affinity bits may meet incompatible nodes: per-node gather below
    const bool factored = NXM_FAST && !(cpic && paff != 0u);
#else
    const bool factored = NXM_FAST;
#endif
    if ((flags & PFLAG_ENABLED) && factored) {
        // Same sums, factored: with dpt_i = ref + s_i dx,
        //   grad = inv_d (v (x) ref + dx [Sx Sy Sz]),  S_a = sum_i w_i v_i s_i,a
        //   vgd  = inv_d (v . ref + dx (Sx.x + Sy.y + Sz.z))
        // so each node costs one weight product and (1 + nonzero s) FMA pairs:
        // the x, y components accumulate as packed f32x2 (FFMA2), z on its own.
        const float inv_dx = prm.inv_dx;
        const v3 ref = assoc_cell_of(dx, pt) * dx - pt;
        const v3 wx = kernel_eval_all(-ref.x * inv_dx);
        const v3 wy = kernel_eval_all(-ref.y * inv_dx);
        const v3 wz = kernel_eval_all(-ref.z * inv_dx);
        const CellInfo ci = cell_info(dx, pt);
        const uint32_t packed = ci.ax + 6u * ci.ay + 36u * ci.az;
        float2 vxy = make_float2(0.f, 0.f), sxxy = vxy, syxy = vxy, szxy = vxy;
        float vz = 0.f, sxz = 0.f, syz = 0.f, szz = 0.f;
#pragma unroll
        for (int sz = 0; sz < 3; ++sz) {
#pragma unroll
            for (int sy = 0; sy < 3; ++sy) {
                const float wyz = vget(wy, sy) * vget(wz, sz);
#pragma unroll
                for (int sx = 0; sx < 3; ++sx) {
                    const float4 h = halo[packed + (uint32_t)(sx + 6 * sy + 36 * sz)];
                    const float2 hxy = make_float2(h.x, h.y);
                    const float w = vget(wx, sx) * wyz;
                    vxy = __ffma2_rn(make_float2(w, w), hxy, vxy);
                    vz = fmaf(w, h.z, vz);
                    if (sx) {
                        const float ws = w * (float)sx;
                        sxxy = __ffma2_rn(make_float2(ws, ws), hxy, sxxy);
                        sxz = fmaf(ws, h.z, sxz);
                    }
                    if (sy) {
                        const float ws = w * (float)sy;
                        syxy = __ffma2_rn(make_float2(ws, ws), hxy, syxy);
                        syz = fmaf(ws, h.z, syz);
                    }
                    if (sz) {
                        const float ws = w * (float)sz;
                        szxy = __ffma2_rn(make_float2(ws, ws), hxy, szxy);
                        szz = fmaf(ws, h.z, szz);
                    }
                }
            }
        }
        velocity = mk(vxy.x, vxy.y, vz);
        const v3 sxv = mk(sxxy.x, sxxy.y, sxz), syv = mk(syxy.x, syxy.y, syz), szv = mk(szxy.x, szxy.y, szz);
        grad = (outer(velocity, ref) + mkm(sxv, syv, szv) * dx) * inv_d;
        vgd = (dot(velocity, ref) + dx * (sxv.x + syv.y + szv.z)) * inv_d;
    } else if (flags & PFLAG_ENABLED) {
        const v3 ref = assoc_cell_of(dx, pt) * dx - pt;
        const v3 w0 = kernel_eval_all(-ref.x / dx);
        const v3 w1 = kernel_eval_all(-ref.y / dx);
        const v3 w2 = kernel_eval_all(-ref.z / dx);
        const CellInfo ci = cell_info(dx, pt);
        const uint32_t packed = ci.ax + 6u * ci.ay + 36u * ci.az;
#pragma unroll
        for (int i = 0; i < 27; ++i) {
            int sx, sy, sz;
            nbh_shift(i, sx, sy, sz);
            const uint32_t hid = packed + (uint32_t)(sx + 6 * sy + 36 * sz);
            const float4 h = halo[hid];
            v3 cv = mk(h.x, h.y, h.z);
            const v3 dpt = ref + mk((float)sx, (float)sy, (float)sz) * dx;
#if NXM_CPIC
            if (cpic) {
                // g2p.rs:206-235: an incompatible node gives its second velocity,
                // projected by its closest body's boundary condition
                const uint2 nc = cx.halo_cdf[hid];
                if (!aff_compatible(paff, nc.x)) {
                    const float4 hi = cx.halo_inc[hid];
                    cv = mk(hi.x, hi.y, hi.z);
                    if (nc.y != NONE) {
                        const DevCollider& c = cx.cols[nc.y];
                        const v3 cell_center = dpt + pt;
                        const v3 bv = col_vel_at(c, cell_center);
                        cv = bv + bc_project(c.bc_type, c.bc_friction * bfric, cv - bv, pnormal);
                    }
                }
            }
#endif
            const float weight = vget(w0, sx) * vget(w1, sy) * vget(w2, sz);
            velocity = velocity + cv * weight;
            grad = grad + outer(cv, dpt) * (weight * inv_d);
            vgd += weight * inv_d * dot(cv, dpt);
        }
#if NXM_CPIC
        if (cpic)  // g2p.rs:248-262: velocity of every body the particle has affinity with
            for (uint32_t ic = 0; ic < 16u && ic < cx.ncols; ++ic)
                if (paff & (1u << ic)) rigid_vel = rigid_vel + col_vel_at(cx.cols[ic], pt);
#endif
    }
#if NXM_CPIC
    if (cpic) P.pcdf[3u * src + 1u] = make_float4(rigid_vel.x, rigid_vel.y, rigid_vel.z, crec1.w);
#endif

    // ---- particle update (particle_update.rs:60-201, non-CPIC: Cdf = 0)
    m3 F = mkm(mk(d0.x, d0.y, d0.z), mk(d1.x, d1.y, d1.z), mk(d2.x, d2.y, d2.z));
    const float init_volume = d0.w, damping = d1.w;
    const uint32_t mid = __float_as_uint(d2.w);
    const Material& mat = P.materials[mid];
    const uint32_t tag = mat.tag;

    v3 v = velocity;
#if NXM_CPIC
    // particle_update.rs:98-102: reproject a penetrating particle
    if (cpic && crec0.w < -0.05f * dx) v = rigid_vel + bc_project(BC_SLIP, 0.0f, v - rigid_vel, pnormal);
#endif
    const float vl = length(v);
    if (vl > dx / dt) v = ((v / vl) * dx) / dt;
    if (NXM_FAST) v = v * (1.0f / (1.0f + damping * dt));  // one division instead of three
    else v = v / (1.0f + damping * dt);
    if (flags & PFLAG_FIXED) v = splat(0.f);
    const v3 np_ = pt + v * dt;
#if NXM_CPIC
    if (cpic && crec0.w < -0.05f * dx) {  // particle_update.rs:132-136 penalty, PENALTY_COEFF = 1e3
        const float corrected = fmaxf(crec0.w, -0.3f * dx);
        v = v + pnormal * (dt * -corrected * 1.0e3f);
    }
#endif
    // The new position, velocity and block key follow from the gather alone:
    // written ahead of the constitutive update (fewer values live across it);
    // a particle that the check after it disables is rewritten there.
    const bool nan = (np_.x != np_.x) || (np_.y != np_.y) || (np_.z != np_.z);
    kr[0] = make_float4(np_.x, np_.y, np_.z, mass);
    kr[1] = make_float4(v.x, v.y, v.z, __uint_as_float(flags));
    {
        const CellInfo nc = cell_info(dx, np_);
        P.pcode[dst] = make_uint2(pack_key(nc.bx + key_off.x, nc.by + key_off.y, nc.bz + key_off.z),
                                  nc.ax | (nc.ay << 2) | (nc.az << 4));
    }
    const m3 A = grad;
    if (tag != MODEL_FLUID) {
        F = F + (A * dt) * F;
    } else {
        const float fd0 = F.c0.x;
        float rate = vgd * dt / 3.0f;
        rate = rclamp(rate, -0.1f, 0.1f);
        const float nd = rclamp(fd0 + rate * fd0, 0.5f, 2.0f);
        F = diag(splat(nd));
    }
    float st[4] = {0.f, 0.f, 0.f, 0.f};
    if (mat.has_state) {
        float4 s4 = P.pstate[src];
        st[0] = s4.x; st[1] = s4.y; st[2] = s4.z; st[3] = s4.w;
    }
    m3 aff;
    if (stash && tag != MODEL_FLUID) {
        // m A waits in this thread's shared-memory slots (stride kG2pThreads) across
        // the model update instead of in registers
        const m3 am = A * mass;
        const float* e = &am.c0.x;
#pragma unroll
        for (int i = 0; i < 9; ++i) stash[kG2pThreads * i] = e[i];
        const m3 tau = model_update<NXM_FAST>(tag, mat.w, st, F, mzero());
        float r[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) r[i] = stash[kG2pThreads * i];
        aff = mkm(mk(r[0], r[1], r[2]), mk(r[3], r[4], r[5]), mk(r[6], r[7], r[8])) -
              tau * (init_volume * inv_d * dt);
    } else {
        const m3 tau = model_update<NXM_FAST>(tag, mat.w, st, F, A);
        aff = A * mass - tau * (init_volume * inv_d * dt);
    }
    if (nan || !(det(F) > 0.0f)) {  // disabled: rewrite what was written ahead
        flags &= ~PFLAG_ENABLED;
        F = mident();
        aff = mzero();
        // the fast build always writes to the other buffer: the old position
        // is re-read there instead of staying live across the model update
        const v3 op = NXM_FAST ? mk(P.kin[src].x, P.kin[src].y, P.kin[src].z) : pt;
        kr[0] = make_float4(op.x, op.y, op.z, 0.f);
        kr[1] = make_float4(0.f, 0.f, 0.f, __uint_as_float(flags));
        const CellInfo oc = cell_info(dx, op);
        P.pcode[dst] = make_uint2(pack_key(oc.bx + key_off.x, oc.by + key_off.y, oc.bz + key_off.z),
                                  oc.ax | (oc.ay << 2) | (oc.az << 4));
    }
    kr[2] = make_float4(aff.c0.x, aff.c0.y, aff.c0.z, vgd);
    kr[3] = make_float4(aff.c1.x, aff.c1.y, aff.c1.z, 0.f);
    kr[4] = make_float4(aff.c2.x, aff.c2.y, aff.c2.z, 0.f);
    float4* dw = reinterpret_cast<float4*>(&P.def_out[dst]);
    dw[0] = make_float4(F.c0.x, F.c0.y, F.c0.z, init_volume);
    dw[1] = make_float4(F.c1.x, F.c1.y, F.c1.z, damping);
    dw[2] = make_float4(F.c2.x, F.c2.y, F.c2.z, d2.w);
    if (mat.has_state) P.pstate_out[dst] = make_float4(st[0], st[1], st[2], st[3]);
    if (P.pid_in) P.pid_out[dst] = P.pid_in[src];
}

// dynamics/body.rs Velocity::integrate for one-way coupled bodies
// (rigid_impulses.rs:66-140 with zero impulse and zero inverse mass): the
// pose of every collider the step moves (all, at most 16, or every scene's
// in batched mode) advances by its velocities over dt.  Run by the first
// threads of the G2P launch, one collider each: nothing in G2P reads a
// collider's rotation or translation (the body velocities it reads use the
// centre of mass refreshed at the start of the step), and the next reader is
// the next step's sort.
__device__ __forceinline__ void integrate_colliders(const DevPtrs& P, const Params& prm) {
    const uint32_t ncol = prm.scene_blocks ? prm.ncol : min(prm.ncol, (uint32_t)MAX_COLLIDERS);
    const float dt = prm.dt;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < ncol; i += gridDim.x * blockDim.x) {
        DevCollider& c = P.colliders[i];
        const quat q = quat{c.rot[0], c.rot[1], c.rot[2], c.rot[3]};
        const v3 tra = mk(c.tra[0], c.tra[1], c.tra[2]);
        const v3 init_com = qrot(q, mk(c.local_com[0], c.local_com[1], c.local_com[2])) + tra;
        const v3 sa = mk(c.angvel[0], c.angvel[1], c.angvel[2]) * dt;
        const float ang = length(sa);
        quat dq;
        if (ang == 0.f) {
            dq = quat{0.f, 0.f, 0.f, 1.f};
        } else {
            const v3 ax = sa / ang;
            const float sh = sinf(ang * 0.5f), ch = cosf(ang * 0.5f);
            dq = quat{ax.x * sh, ax.y * sh, ax.z * sh, ch};
        }
        const v3 dl = mk(c.linvel[0], c.linvel[1], c.linvel[2]) * dt;
        const v3 nt = (init_com + qrot(dq, tra - init_com)) + dl;
        quat nr;
        nr.w = dq.w * q.w - dq.x * q.x - dq.y * q.y - dq.z * q.z;
        nr.x = dq.w * q.x + dq.x * q.w + dq.y * q.z - dq.z * q.y;
        nr.y = dq.w * q.y - dq.x * q.z + dq.y * q.w + dq.z * q.x;
        nr.z = dq.w * q.z + dq.x * q.y - dq.y * q.x + dq.z * q.w;
        const float rl = 1.0f / sqrtf(nr.x * nr.x + nr.y * nr.y + nr.z * nr.z + nr.w * nr.w);
        c.rot[0] = nr.x * rl; c.rot[1] = nr.y * rl; c.rot[2] = nr.z * rl; c.rot[3] = nr.w * rl;
        c.tra[0] = nt.x; c.tra[1] = nt.y; c.tra[2] = nt.z;
    }
}

// End of a G2P launch: when reordering, the particles the sort could not
// place (their block was not created: capacity or hash overflow, reported in
// the status word) are copied unchanged to the slots after the sorted ones;
// then the cached block keys are marked valid.
__device__ __forceinline__ void g2p_finish(const DevPtrs& P, const Params& prm) {
    if (P.pid_in) {
        const uint32_t n = prm.n, sl = __ldcg(&P.counters->sorted_len);
        for (uint32_t p = sl < n ? blockIdx.x * blockDim.x + threadIdx.x : n; p < n; p += gridDim.x * blockDim.x) {
            if (__ldcg(&P.phdr[p]) != NONE) continue;
            const uint32_t dst = sl + atomicAdd(&P.counters->unsorted, 1u);
            if (dst >= n) continue;  // not reached: exactly n - sl particles have no header
            const float4* ks = reinterpret_cast<const float4*>(&P.kin[p]);
            float4* kd = reinterpret_cast<float4*>(&P.kin_out[dst]);
#pragma unroll
            for (int w = 0; w < 5; ++w) kd[w] = ks[w];
            const float4* ds = reinterpret_cast<const float4*>(&P.def[p]);
            float4* dd = reinterpret_cast<float4*>(&P.def_out[dst]);
#pragma unroll
            for (int w = 0; w < 3; ++w) dd[w] = ds[w];
            P.pstate_out[dst] = P.pstate[p];
            P.pid_out[dst] = P.pid_in[p];
            const CellInfo nc = cell_info(prm.dx, mk(ks[0].x, ks[0].y, ks[0].z));
            const int3 o = prm.scene_blocks ? scene_base_of(prm, P.pscene[P.pid_in[p]]) : make_int3(0, 0, 0);
            P.pcode[dst] = make_uint2(pack_key(nc.bx + o.x, nc.by + o.y, nc.bz + o.z),
                                      nc.ax | (nc.ay << 2) | (nc.az << 4));
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) P.counters->codes_valid = 1u;
}

#ifndef NXM_G2P_MIN_CTAS
#define NXM_G2P_MIN_CTAS 4  // CTAs per SM the register budget is sized for
#endif

// One CTA per primary block (ids [0, num_primary); the other blocks hold no
// particles), grid-stride: the halo of the block and its +1 neighbours is
// staged in shared memory, then each thread gathers and updates one of the
// block's primary particles.  The next block's header is loaded one block
// ahead, and each thread's first particle is fetched alongside the halo so
// that the two dependent load chains overlap.  When reordering, sorted entry
// j = first + k goes to output slot j; particles the sort could not place
// (their block was not created: capacity or hash overflow, reported in the
// status word) are copied unchanged to the slots after the sorted ones.
#ifndef NXM_G2P_STASH
#define NXM_G2P_STASH 1  // m A waits in shared memory across the model update (fast build)
#endif
// Below prm.range_min_fill particles a block on average (64 unless tuned), a
// run of the fast G2P (k_g2p_range) would span more blocks than one pass
// stages: such a launch (decided on the device from this step's counts, the
// same in every CTA) runs the per-block loop, where the blocks of a small
// sparse scene are side by side on many CTAs instead of passes in a row on a
// few.
__device__ __forceinline__ bool g2p_sparse(const DevPtrs& P, const Params& prm) {
    const uint32_t nbp = min(__ldcg(&P.counters->num_primary), __ldcg(&P.counters->num_blocks));
    const uint32_t len = min(__ldcg(&P.counters->sorted_len), prm.n);
    return (uint64_t)len < (uint64_t)prm.range_min_fill * nbp;
}

// The per-block loop: one CTA per primary block (grid-stride), halo of 216
// nodes in `halo` (CPIC: the incompatible fields and node distance field in
// halo_inc / halo_cdf).
__device__ __forceinline__ void g2p_block_loop(const DevPtrs& P, const Params& prm, float4* halo, float4* halo_inc,
                                               uint2* halo_cdf, volatile float* stash) {
    (void)halo_inc;
    (void)halo_cdf;
    const uint32_t nbp = min(__ldcg(&P.counters->num_primary), __ldcg(&P.counters->num_blocks));
    const uint32_t tid = threadIdx.x;
    const uint32_t ht = tid < 216u ? tid : 0u;  // halo node of this thread
    const uint32_t htx = ht % 6u, hty = (ht / 6u) % 6u, htz = ht / 36u;
    const uint32_t hox = htx >= 4u, hoy = hty >= 4u, hoz = htz >= 4u;
    const uint32_t hoct = hox * 4u + hoy * 2u + hoz;
    const uint32_t hnode = (htx - 4u * hox) + 4u * (hty - 4u * hoy) + 16u * (htz - 4u * hoz);
    uint32_t b = blockIdx.x;
    uint32_t first = 0, np = 0;
    if (b < nbp) {
        first = __ldcg(&P.first[b]);
        np = __ldcg(&P.nprim[b]);
    }
    while (b < nbp) {
        const uint32_t bn = b + gridDim.x;
        uint32_t nfirst = 0, nnp = 0;
        if (bn < nbp) {
            nfirst = __ldcg(&P.first[bn]);
            nnp = __ldcg(&P.nprim[bn]);
        }
        const bool reorder = P.pid_in != nullptr;
        const int3 key_off = prm.scene_blocks ? scene_base_of_block(prm, P.bvid[b]) : make_int3(0, 0, 0);
        uint32_t pid = tid < np ? __ldg(&P.sorted[first + tid]) : NONE;
        const uint32_t hblk = (tid < 216u && hoct != 0u) ? __ldg(&P.nbh[b * NUM_NBH + hoct - 1u]) : b;
        float4 xm = make_float4(0.f, 0.f, 0.f, 0.f), vf = xm;
        if (pid != NONE) {
            const float4* kr = reinterpret_cast<const float4*>(&P.kin[pid]);
            xm = kr[0];
            vf = kr[1];
        }
        if (tid < 216u) {
            float4 nd = make_float4(0.f, 0.f, 0.f, 0.f);
            if (hblk != NONE) nd = P.nodes[hblk * 64u + hnode];
            halo[tid] = make_float4(nd.x, nd.y, nd.z, 0.f);
        }
        for (uint32_t t = tid + blockDim.x; t < 216u; t += blockDim.x) halo[t] = halo_node(P, b, t);
        CpicCtx cx{nullptr, nullptr, P.colliders, 0u};
#if NXM_CPIC
        // A halo whose nodes carry no affinity bit gave every particle of the
        // block an empty affinity and a zero distance record (g2p_cdf): all
        // nodes are compatible, no body velocity enters and the record stays
        // zero, so the block runs the plain transfer (halo_cdf left null).
        bool cpic_block = false;
        if (prm.use_cpic) {
            uint32_t any = 0u;
            for (uint32_t t = tid; t < 216u; t += blockDim.x) {
                const uint32_t tx = t % 6u, ty = (t / 6u) % 6u, tz = t / 36u;
                const uint32_t ox = tx >= 4u, oy = ty >= 4u, oz = tz >= 4u;
                const uint32_t oct = ox * 4u + oy * 2u + oz;
                const uint32_t blk = oct == 0 ? b : P.nbh[b * NUM_NBH + oct - 1u];
                const uint32_t node = (tx - 4u * ox) + 4u * (ty - 4u * oy) + 16u * (tz - 4u * oz);
                const uint4 nc = blk == NONE ? make_uint4(0u, 0u, NONE, 0u) : P.ncdf[blk * 64u + node];
                halo_cdf[t] = make_uint2(nc.y, nc.z);
                any |= nc.y;
            }
            cpic_block = __syncthreads_or((int)(any & 0x0000FFFFu)) != 0;
        }
        if (cpic_block) {
            for (uint32_t t = tid; t < 216u; t += blockDim.x) {
                const uint32_t tx = t % 6u, ty = (t / 6u) % 6u, tz = t / 36u;
                const uint32_t ox = tx >= 4u, oy = ty >= 4u, oz = tz >= 4u;
                const uint32_t oct = ox * 4u + oy * 2u + oz;
                const uint32_t blk = oct == 0 ? b : P.nbh[b * NUM_NBH + oct - 1u];
                const uint32_t node = (tx - 4u * ox) + 4u * (ty - 4u * oy) + 16u * (tz - 4u * oz);
                halo_inc[t] = blk == NONE ? make_float4(0.f, 0.f, 0.f, 0.f) : P.nodes_inc[blk * 64u + node];
            }
            cx.halo_inc = halo_inc;
            cx.halo_cdf = halo_cdf;
            if (prm.scene_blocks) {
                const uint32_t sid = scene_of_block(prm, P.bvid[b]);
                const uint2 r = sid != NONE ? P.scene_cols[sid] : make_uint2(0u, 0u);
                cx.cols = P.colliders + r.x;
                cx.ncols = min(r.y, (uint32_t)MAX_COLLIDERS);
            } else {
                cx.ncols = min(prm.ncol, (uint32_t)MAX_COLLIDERS);
            }
        }
#endif
        __syncthreads();
        for (uint32_t k = tid; k < np; k += blockDim.x) {
            if (k != tid) {
                pid = P.sorted[first + k];
                const float4* kr = reinterpret_cast<const float4*>(&P.kin[pid]);
                xm = kr[0];
                vf = kr[1];
            }
#if NXM_CPIC
            if (cx.halo_cdf) g2p_particle<true>(P, prm, halo, pid, reorder ? first + k : pid, xm, vf, key_off, cx, stash);
            else
#endif
                g2p_particle<false>(P, prm, halo, pid, reorder ? first + k : pid, xm, vf, key_off, cx, stash);
        }
        __syncthreads();
        b = bn;
        first = nfirst;
        np = nnp;
    }
}

__global__ void __launch_bounds__(kG2pThreads, NXM_G2P_MIN_CTAS) k_g2p_update(DevPtrs P) {
    __shared__ float4 halo[216];
#if NXM_G2P_STASH
    __shared__ float stash_mem[9 * kG2pThreads];
    volatile float* stash = NXM_FAST ? stash_mem + threadIdx.x : nullptr;
#else
    volatile float* stash = nullptr;
#endif
#if NXM_CPIC
    __shared__ float4 halo_inc[216];
    __shared__ uint2 halo_cdf[216];
#else
    float4* halo_inc = nullptr;
    uint2* halo_cdf = nullptr;
#endif
    const Params prm = *P.params;
    integrate_colliders(P, prm);
    g2p_block_loop(P, prm, halo, halo_inc, halo_cdf, stash);
    g2p_finish(P, prm);
}

#if NXM_FAST && !NXM_CPIC
// ---- bulk (TMA) copies of node blocks into shared memory -------------------
// One elected thread issues 1-D cp.async.bulk copies of whole 1 KB node
// blocks (global memory of this GPU only, no multicast) that complete on an
// mbarrier in shared memory; every thread then waits on the barrier's phase,
// with an iteration limit after which the kernel records
// STATUS_COPY_TIMEOUT instead of waiting on.
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// Waits for the barrier's phase `parity` to complete; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
constexpr uint32_t kCopyWaitLimit = 1u << 20;  // try_wait rounds (each may suspend a few us): over a second

// Stages the 6x6x6 node-velocity halos of blocks [b, b + cnt) into `halo`
// by bulk copies: per group of kTmaGroup blocks, thread 0 copies the 8 node
// blocks each halo draws from (the block and its 7 +1 neighbours; a missing
// one from the zero block after the grid, index block_capacity) into `raw`,
// 8 KB a block, completing on the CTA's barrier; every thread waits for the
// phase, then the CTA rearranges them into halo order.  Ends with a CTA
// barrier.
constexpr uint32_t kTmaGroup = 2;
__device__ __forceinline__ void stage_halos_tma(const DevPtrs& P, uint32_t b, uint32_t cnt, float4* halo, float4* raw,
                                                uint64_t* bar, uint32_t& parity, uint32_t zero_blk) {
    const uint32_t tid = threadIdx.x;
    for (uint32_t g0 = 0; g0 < cnt; g0 += kTmaGroup) {
        const uint32_t gc = min(cnt - g0, kTmaGroup);
        if (tid == 0) {
            // the raw area was last read by the generic proxy (the previous group's rearrangement)
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(bar, gc * 8u * 1024u);
            for (uint32_t j = 0; j < gc; ++j) {
                const uint32_t blk = b + g0 + j;
                uint32_t nb[7];
#pragma unroll
                for (uint32_t o = 0; o < 7; ++o) nb[o] = __ldcg(&P.nbh[blk * NUM_NBH + o]);
                bulk_copy_g2s(raw + (j * 8u) * 64u, P.nodes + (size_t)blk * 64u, 1024u, bar);
#pragma unroll
                for (uint32_t o = 1; o < 8; ++o) {
                    const uint32_t src = nb[o - 1] == NONE ? zero_blk : nb[o - 1];
                    bulk_copy_g2s(raw + (j * 8u + o) * 64u, P.nodes + (size_t)src * 64u, 1024u, bar);
                }
            }
        }
        if (!mbar_wait(bar, parity, kCopyWaitLimit)) {
            if (tid == 0) set_status(P.counters, STATUS_COPY_TIMEOUT);
            mbar_wait(bar, parity, kCopyWaitLimit);  // the copies may still be in flight: wait once more
        }
        parity ^= 1u;
        for (uint32_t t = tid; t < gc * 216u; t += blockDim.x) {
            const uint32_t j = t / 216u, node = t - 216u * j;
            const uint32_t tx = node % 6u, ty = (node / 6u) % 6u, tz = node / 36u;
            const uint32_t ox = tx >= 4u, oy = ty >= 4u, oz = tz >= 4u;
            const uint32_t oct = ox * 4u + oy * 2u + oz;
            const float4 nd = raw[(j * 8u + oct) * 64u + (tx - 4u * ox) + 4u * (ty - 4u * oy) + 16u * (tz - 4u * oz)];
            halo[(g0 + j) * 216u + node] = make_float4(nd.x, nd.y, nd.z, 0.f);
        }
        __syncthreads();  // raw is free again; the halos are complete
    }
}

// The wait above, made to run out: a barrier that expects bytes no copy will
// deliver (nothing is issued), waited on with `limit` rounds; the kernel
// records STATUS_COPY_TIMEOUT and returns with no copy in flight.
__global__ void k_copy_wait_timeout(Counters* counters, uint32_t limit) {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar);
        mbar_expect_tx(&bar, 16u);
    }
    __syncthreads();
    if (!mbar_wait(&bar, 0u, limit) && threadIdx.x == 0) set_status(counters, STATUS_COPY_TIMEOUT);
}

// The fast build's G2P walks the sorted list in runs of kRangeChunk
// positions, one particle per thread, instead of one CTA per block: a block
// holds some 1-600 particles, so per-block rounds of 256 threads run part
// empty (three quarters full on a settled scene); a run fills every thread
// but one run's worth at the end.  The fast path lists no extras, so the
// positions [0, sorted_len) are exactly the primary particles, block after
// block; run c spans the blocks [chunk_blk[c], chunk_blk[c + 1]] (the scan
// records the block of each run's first position; the last run reaches the
// last primary block), usually one or two.  Their halos are staged
// kRangeHalos at a time, and each thread takes its particle's block from the
// header id the sort's count pass stored for it (phdr).  A run's span is
// loaded one run ahead, so that a run's own loads (ids, records, halos) are
// issued together.
//
// A launch over sparse blocks (g2p_sparse) takes one block per unit instead
// (its particles in rounds of 256), through the same loop: a unit is a span
// of blocks whose halos are staged in passes and a range of sorted positions
// the threads step through, so the particle update has one call site.
//
// Halo staging: plain loads by every thread (each node: its block id from the
// neighbour table, then the node, both L2 hits) by default; with
// NXM_G2P_TMA_HALO the bulk copies of stage_halos_tma instead (measured
// slower on the 2 M-particle scene: the rearrangement pass and its barriers
// cost more than the loads they replace).
#ifndef NXM_G2P_TMA_HALO
#define NXM_G2P_TMA_HALO 0
#endif
constexpr uint32_t kRangeHalos = 8;
static_assert(kG2pThreads == kRangeChunk, "one sorted position per thread");
#if NXM_G2P_TMA_HALO
constexpr size_t kG2pRangeSmem = (size_t)kRangeHalos * 216 * 16 + (size_t)kTmaGroup * 8 * 64 * 16 +
                                 (size_t)9 * 4 * kG2pThreads + 16;
#endif
__global__ void __launch_bounds__(kG2pThreads, NXM_G2P_MIN_CTAS) k_g2p_range(DevPtrs P) {
#if NXM_G2P_TMA_HALO
    extern __shared__ float4 g2p_smem[];
    float4* halo = g2p_smem;                 // kRangeHalos x 216 nodes
    float4* raw = halo + kRangeHalos * 216;  // kTmaGroup x 8 node blocks
    float* stash_mem = reinterpret_cast<float*>(raw + kTmaGroup * 8 * 64);
    uint64_t* bar = reinterpret_cast<uint64_t*>(stash_mem + 9 * kG2pThreads);
    if (threadIdx.x == 0) mbar_init(bar);
    __syncthreads();
    uint32_t parity = 0;
    const uint32_t zero_blk = P.params->block_capacity;
#else
    __shared__ float4 halo[kRangeHalos * 216];
    __shared__ float stash_mem[9 * kG2pThreads];
#endif
#if NXM_G2P_STASH
    volatile float* stash = stash_mem + threadIdx.x;
#else
    volatile float* stash = nullptr;
#endif
    const Params prm = *P.params;
    integrate_colliders(P, prm);
    const uint32_t nbp = min(__ldcg(&P.counters->num_primary), __ldcg(&P.counters->num_blocks));
    const uint32_t len = min(__ldcg(&P.counters->sorted_len), prm.n);
    const bool sparse = g2p_sparse(P, prm);
    const uint32_t nunits = !nbp ? 0u : (sparse ? nbp : min((len + kRangeChunk - 1u) / kRangeChunk, P.chunk_cap));
    const uint32_t tid = threadIdx.x;
    const bool reorder = P.pid_in != nullptr;
    const CpicCtx cx{nullptr, nullptr, P.colliders, 0u};
    // unit u: blocks [lo, hi], sorted positions [p0, p1), from two loaded
    // words (dense: the run's first and last block; sparse: first, nprim of
    // the block), loaded one unit ahead
    auto words_of = [&](uint32_t u, uint32_t& a, uint32_t& b) {
        if (sparse) {
            a = __ldcg(&P.first[u]);
            b = __ldcg(&P.nprim[u]);
        } else {
            a = __ldcg(&P.chunk_blk[u]);
            b = u + 1u < nunits ? __ldcg(&P.chunk_blk[u + 1u]) : nbp - 1u;
        }
    };
    uint32_t u = blockIdx.x, wa = 0u, wb = 0u;
    if (u < nunits) words_of(u, wa, wb);
    for (; u < nunits; u += gridDim.x) {
        uint32_t lo, hi, p0, p1;
        if (sparse) {
            lo = hi = u;
            p0 = wa;
            p1 = min(wa + wb, len);
        } else {
            lo = wa;
            hi = min(wb, nbp - 1u);
            p0 = u * kRangeChunk;
            p1 = min(p0 + kRangeChunk, len);
        }
        if (u + gridDim.x < nunits) words_of(u + gridDim.x, wa, wb);
        // this thread's first particle, fetched while the halos load
        uint32_t pid = p0 + tid < p1 ? __ldg(&P.sorted[p0 + tid]) : NONE;
        float4 xm = make_float4(0.f, 0.f, 0.f, 0.f), vf = xm;
        uint32_t blk = lo;
        if (pid != NONE) {
            const float4* kr = reinterpret_cast<const float4*>(&P.kin[pid]);
            xm = kr[0];
            vf = kr[1];
            if (!sparse) blk = __ldcg(&P.phdr[pid]);
        }
        bool pending = pid != NONE;  // dense: this thread's one particle not yet updated
        for (uint32_t b = lo; b <= hi; b += kRangeHalos) {
            const uint32_t cnt = min(hi - b + 1u, kRangeHalos);
#if NXM_G2P_TMA_HALO
            stage_halos_tma(P, b, cnt, halo, raw, bar, parity, zero_blk);
#else
            for (uint32_t t = tid; t < cnt * 216u; t += kG2pThreads) {
                const uint32_t i = t / 216u;
                halo[t] = halo_node(P, b + i, t - 216u * i);
            }
            __syncthreads();
#endif
            // dense: one position per thread; sparse: the block's positions in rounds
            for (uint32_t p = p0 + tid; p < p1; p += kG2pThreads) {
                if (p != p0 + tid) {
                    pid = __ldg(&P.sorted[p]);
                    const float4* kr = reinterpret_cast<const float4*>(&P.kin[pid]);
                    xm = kr[0];
                    vf = kr[1];
                }
                if (blk >= b && blk - b < cnt) {
                    const int3 key_off =
                        prm.scene_blocks ? scene_base_of_block(prm, P.bvid[blk]) : make_int3(0, 0, 0);
                    g2p_particle<false>(P, prm, halo + 216u * (blk - b), pid, reorder ? p : pid, xm, vf, key_off, cx,
                                 stash);
                    pending = false;
                }
            }
            __syncthreads();
        }
        if (!sparse && pending) set_status(P.counters, STATUS_MISSING_BLOCK);  // not reached: a run holds its blocks
    }
    g2p_finish(P, prm);
}
#endif

}  // namespace

#if NXM_FAST && !NXM_CPIC
void launch_copy_wait_timeout(Counters* counters, uint32_t limit, cudaStream_t s) {
    k_copy_wait_timeout<<<1, 32, 0, s>>>(counters, limit);
}
#endif

void launch_grid_update(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s) {
    k_grid_update<<<c.sm_count * (int)c.t.grid_ctas, 256, 0, s>>>(P);
}

int launch_g2p_update(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s) {
#if NXM_FAST && !NXM_CPIC && !defined(NXM_G2P_PER_BLOCK)
    if (P.chunk_blk) {  // runs of the sorted list, or one block per unit over sparse blocks
#if NXM_G2P_TMA_HALO
        cudaFuncSetAttribute(k_g2p_range, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kG2pRangeSmem);
        cudaFuncSetAttribute(k_g2p_range, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        k_g2p_range<<<c.sm_count * (int)min(c.t.g2p_ctas, (uint32_t)NXM_G2P_MIN_CTAS), kG2pThreads, kG2pRangeSmem,
                      s>>>(P);
#else
        k_g2p_range<<<c.sm_count * (int)min(c.t.g2p_ctas, (uint32_t)NXM_G2P_MIN_CTAS), kG2pThreads, 0, s>>>(P);
#endif
        return 1;
    }
#endif
    k_g2p_update<<<c.sm_count * NXM_G2P_MIN_CTAS, kG2pThreads, 0, s>>>(P);
    return 1;
}

}  // namespace NXM_NS
}  // namespace nxm
