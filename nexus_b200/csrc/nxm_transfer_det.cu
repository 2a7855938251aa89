// Deterministic-mode transfers, built with --fmad=false: the reference's
// atomic-free, gather-form P2G (solver/p2g.rs:64-351, USE_CPIC = false) with
// its chunking, z-slab culling and summation order, plus the grid update and
// fused G2P + particle update of nxm_transfer.inc.cuh.  Given the canonical
// sort order these reproduce the CPU oracle's f32 arithmetic operation by
// operation (up to the last bits of logf/expf/sinf).
#define NXM_NS exact
#define NXM_FAST false
#define NXM_CPIC 1
#include "nxm_transfer.inc.cuh"

namespace nxm {
namespace exact {
namespace {

// One CTA of 64 threads (one per node of the block, tid = x + 4y + 16z).
__global__ void __launch_bounds__(64) k_p2g_gather(DevPtrs P) {
    __shared__ float spx[64], spy[64], spz[64];
    __shared__ float smx[64], smy[64], smz[64], smass[64];
    __shared__ float saff[9][64];
    __shared__ int szkey[64];
    __shared__ uint32_t safn[64];  // particle affinity bits (CPIC)
    const bool cpic = P.params->use_cpic != 0;
    const float dx = P.params->dx;
    const float inv_cell_width = 1.0f / dx;
    const uint32_t nb = P.counters->num_blocks;
    const uint32_t tid = threadIdx.x;
    const int tx = (int)(tid & 3u), ty = (int)((tid >> 2) & 3u), tz = (int)(tid >> 4);
    for (uint32_t b = blockIdx.x; b < nb; b += gridDim.x) {
        int4 vid = P.bvid[b];
        {
            const int3 o = scene_base_of_block(*P.params, vid);  // scene-local block coordinates
            vid.x -= o.x; vid.y -= o.y; vid.z -= o.z;
        }
        const v3 cell_pos = mk((float)(vid.x * 4 + tx), (float)(vid.y * 4 + ty), (float)(vid.z * 4 + tz)) * dx;
        const uint32_t first = P.first[b];
        const uint32_t num = P.nwx[b];
        const uint32_t last = first + num;
        const uint32_t primaries_end = first + P.nprim[b];
        const uint32_t nchunks = (num + 63u) / 64u;
        v3 acc_mv = splat(0.f), acc_mvi = splat(0.f);
        float acc_mass = 0.f, acc_massi = 0.f;
        const uint32_t node_aff = cpic ? P.ncdf[b * 64u + tid].y : 0u;
        for (uint32_t chunk = 0; chunk < nchunks; ++chunk) {
            const uint32_t chunk_base = first + chunk * 64u;
            __syncthreads();
            const uint32_t load_idx = chunk_base + tid;
            if (load_idx < last) {
                const uint32_t pid = P.sorted[load_idx];
                const float4* kr = reinterpret_cast<const float4*>(&P.kin[pid]);
                const float4 xm = kr[0], vf = kr[1];
                const v3 pt = mk(xm.x, xm.y, xm.z);
                const v3 ac = assoc_cell_of(dx, pt);
                int zk = f2i_sat(ac.z) - vid.z * 4;
                szkey[tid] = zk < -2 ? -2 : zk;
                safn[tid] = cpic ? __float_as_uint(P.pcdf[3u * pid + 1u].w) : 0u;
                if (__float_as_uint(vf.w) & PFLAG_ENABLED) {
                    const float4 c0 = kr[2], c1 = kr[3], c2 = kr[4];
                    const float m = xm.w;
                    spx[tid] = pt.x; spy[tid] = pt.y; spz[tid] = pt.z;
                    smx[tid] = vf.x * m; smy[tid] = vf.y * m; smz[tid] = vf.z * m;
                    smass[tid] = m;
                    saff[0][tid] = c0.x; saff[1][tid] = c0.y; saff[2][tid] = c0.z;
                    saff[3][tid] = c1.x; saff[4][tid] = c1.y; saff[5][tid] = c1.z;
                    saff[6][tid] = c2.x; saff[7][tid] = c2.y; saff[8][tid] = c2.z;
                } else {
                    spx[tid] = 0.f; spy[tid] = 0.f; spz[tid] = 0.f;
                    smx[tid] = 0.f; smy[tid] = 0.f; smz[tid] = 0.f;
                    smass[tid] = 0.f;
#pragma unroll
                    for (int q = 0; q < 9; ++q) saff[q][tid] = 0.f;
                }
            }
            __syncthreads();
            const uint32_t chunk_len = min(last - chunk_base, 64u);
            int zmin = szkey[0];
            int zmax = szkey[chunk_len - 1];
            if (primaries_end > chunk_base && primaries_end < chunk_base + chunk_len) {
                const uint32_t bb = primaries_end - chunk_base;
                zmin = min(zmin, szkey[bb]);
                zmax = max(zmax, szkey[bb - 1]);
            }
            const bool in_range = tz >= zmin && tz <= zmax + 2;
            const uint32_t culled = in_range ? chunk_len : 0u;
            for (uint32_t p = 0; p < culled; ++p) {
                const v3 dpt = cell_pos - mk(spx[p], spy[p], spz[p]);
                const float weight = kernel_eval(dpt.x * inv_cell_width) * kernel_eval(dpt.y * inv_cell_width) *
                                     kernel_eval(dpt.z * inv_cell_width);
                if (weight != 0.f) {
                    const m3 A = mkm(mk(saff[0][p], saff[1][p], saff[2][p]), mk(saff[3][p], saff[4][p], saff[5][p]),
                                     mk(saff[6][p], saff[7][p], saff[8][p]));
                    const v3 vel_contribution = (A * dpt + mk(smx[p], smy[p], smz[p])) * weight;
                    const float mass_contribution = smass[p] * weight;
                    // p2g.rs:268-305: an incompatible particle feeds the node's second field
                    if (cpic && !aff_compatible(safn[p], node_aff)) {
                        acc_mvi = acc_mvi + vel_contribution;
                        acc_massi += mass_contribution;
                    } else {
                        acc_mv = acc_mv + vel_contribution;
                        acc_mass += mass_contribution;
                    }
                }
            }
        }
        P.nodes[b * 64u + tid] = make_float4(acc_mv.x, acc_mv.y, acc_mv.z, acc_mass);
        if (cpic) P.nodes_inc[b * 64u + tid] = make_float4(acc_mvi.x, acc_mvi.y, acc_mvi.z, acc_massi);
        __syncthreads();
    }
}

// CFL timestep bound (solver/timestep_bound.rs:59-115): per enabled
// particle, the model's sound-speed bound (models/default.rs:268-343,
// models/utils.rs:157-175) and the velocity + APIC bound, reduced with an
// atomic min on the fixed-point value (dt * 1e12) as u32.  Built without
// multiply-add contraction, so the value matches the f32 oracle's.
__device__ __forceinline__ float sound_speed_bound(float alpha, float bulk, float shear, float density0,
                                                   float def_grad_det, v3 vel, float cell_width) {
    const float curr_density = density0 / fmaxf(def_grad_det, 1.0e-6f);
    const float sound_speed = sqrtf((bulk + shear * 4.0f / 3.0f) / curr_density);
    const float max_speed = fmaxf(length(vel), sound_speed);
    return alpha * cell_width / max_speed;
}
// linear_elasticity.rs:58-80 / neo_hookean_elasticity.rs:43-65: words lambda, mu, cfl at w[o..o+3)
__device__ __forceinline__ float elastic_bound(const float* w, int o, float hardening, float density0, float jdet,
                                               v3 vel, float cw) {
    const float bulk = w[o] + 2.0f * w[o + 1] / 3.0f;  // utils.rs:34-36
    const float shear = w[o + 1];                      // utils.rs:28-30
    return sound_speed_bound(w[o + 2], bulk * hardening, shear * hardening, density0, jdet, vel, cw);
}

__global__ void __launch_bounds__(256) k_timestep_bound(DevPtrs P) {
    const uint32_t n = P.params->n;
    const float cw = P.params->dx;
    uint32_t best = 0xFFFFFFFFu;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const float4* kr = reinterpret_cast<const float4*>(&P.kin[p]);
        const float4 xm = kr[0], vf = kr[1];
        if (!(__float_as_uint(vf.w) & PFLAG_ENABLED)) continue;
        const float4 c0 = kr[2], c1 = kr[3], c2 = kr[4];
        const float4* dr = reinterpret_cast<const float4*>(&P.def[p]);
        const float4 d0 = dr[0], d1 = dr[1], d2 = dr[2];
        const m3 F = mkm(mk(d0.x, d0.y, d0.z), mk(d1.x, d1.y, d1.z), mk(d2.x, d2.y, d2.z));
        const Material& mat = P.materials[__float_as_uint(d2.w)];
        const float* w = mat.w;
        const float mass = xm.w;
        const float density0 = mass / d0.w;
        const float jdet = det(F);
        const v3 vel = mk(vf.x, vf.y, vf.z);
        float dt;
        switch (mat.tag) {
        case MODEL_ELASTIC_LINEAR:
        case MODEL_ELASTIC_NEO_HOOKEAN: dt = elastic_bound(w, 0, 1.0f, density0, jdet, vel, cw); break;
        case MODEL_SAND_LINEAR:
        case MODEL_SAND_NEO_HOOKEAN: dt = elastic_bound(w, 10, 1.0f, density0, jdet, vel, cw); break;
        case MODEL_FLUID:  // fluid.rs:88-108: bulk modulus * gamma, no shear
            dt = sound_speed_bound(w[3], w[0] * w[1], 0.0f, density0, jdet, vel, cw);
            break;
        case MODEL_SNOW: {  // snow.rs:77-79: hardening from the particle's plastic det
            const float hard = expf(w[3] * (1.0f - P.pstate[p].x));
            dt = elastic_bound(w, 4, hard, density0, jdet, vel, cw);
            break;
        }
        default: dt = 0.0f; break;
        }
        const v3 a0 = mk(c0.x, c0.y, c0.z), a1 = mk(c1.x, c1.y, c1.z), a2 = mk(c2.x, c2.y, c2.z);
        const float na2 = dot(a0, a0) + dot(a1, a1) + dot(a2, a2);
        const float d = (cw * cw) / 4.0f;
        const float norm_b = d * sqrtf(na2) / mass;
        const float apic_v = norm_b * 6.0f * sqrtf(3.0f) / cw;
        const float v = length(vel) + apic_v;
        dt = fminf(dt, cw / v);
        best = min(best, __float2uint_rz(dt * 1.0e12f));  // saturating, NaN -> 0, as Rust `as u32`
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xFFFFFFFFu, best, o));
    if ((threadIdx.x & 31u) == 0 && best != 0xFFFFFFFFu) atomicMin(&P.counters->dt_bound, best);
}

// ---- CPIC distance fields -----------------------------------------------------

// Colliders a block sees: all (at most 16), or its scene's in batched mode.
__device__ __forceinline__ const DevCollider* block_colliders(const DevPtrs& P, const Params& prm, int4 vid,
                                                             uint32_t* n) {
    if (prm.scene_blocks) {
        const uint32_t sid = scene_of_block(prm, vid);
        const uint2 r = sid != NONE ? P.scene_cols[sid] : make_uint2(0u, 0u);
        *n = min(r.y, (uint32_t)MAX_COLLIDERS);
        return P.colliders + r.x;
    }
    *n = min(prm.ncol, (uint32_t)MAX_COLLIDERS);
    return P.colliders;
}

// solver/grid_update_cdf.rs:18-58: per node, every ball / cuboid / capsule
// within 1.5 dx (or containing the node) sets its affinity bit (and its sign
// bit when inside); the closest by unsigned distance is kept.  Trimeshes
// reach the node field through their rigid particles (k_p2g_cdf).
__global__ void __launch_bounds__(256) k_grid_update_cdf(DevPtrs P) {
    const Params prm = *P.params;
    const float dx = prm.dx, cap = dx * 1.5f;
    const uint32_t total = P.counters->num_blocks * 64u;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const uint32_t b = t >> 6, k = t & 63u;
        int4 vid = P.bvid[b];
        uint32_t ncol;
        const DevCollider* cols = block_colliders(P, prm, vid, &ncol);
        const int3 o = scene_base_of_block(prm, vid);
        vid.x -= o.x; vid.y -= o.y; vid.z -= o.z;
        const v3 point = mk((float)(vid.x * 4 + (int)(k & 3u)), (float)(vid.y * 4 + (int)((k >> 2) & 3u)),
                            (float)(vid.z * 4 + (int)(k >> 4))) * dx;
        float dist = MAX_FLT;
        uint32_t aff = 0u, closest = NONE;
        // the warp's 32 nodes share one block: its analytic colliders in reach
        const uint32_t near = colliders_near_block(P, cols, ncol, dx, vid, true);
        for (uint32_t i = 0; i < ncol; ++i) {
            const DevCollider& c = cols[i];
            if (c.type == SHAPE_TRIMESH || !(near & (1u << i))) continue;
            const quat q = quat{c.rot[0], c.rot[1], c.rot[2], c.rot[3]};
            const v3 tra = mk(c.tra[0], c.tra[1], c.tra[2]);
            const v3 local = qrot(qconj(q), point - tra);
            Proj pr;
            if (c.type == SHAPE_BALL) pr = ball_project_local(c.a[0], local);
            else if (c.type == SHAPE_CUBOID) pr = cuboid_project_local(mk(c.a[0], c.a[1], c.a[2]), local);
            else if (c.type == SHAPE_CAPSULE)
                pr = capsule_project_local(mk(c.a[0], c.a[1], c.a[2]), mk(c.b[0], c.b[1], c.b[2]), c.b[3], local);
            else { pr.point = local; pr.inside = false; }
            pr.point = qrot(q, pr.point) + tra;
            const v3 dpt = pr.point - point;
            const v3 ad = vabs(dpt);
            if (pr.inside || (ad.x <= cap && ad.y <= cap && ad.z <= cap)) {
                const float d = length(dpt);
                if (d < dist) {
                    closest = i;
                    dist = d;
                }
                aff |= (pr.inside ? 0x00010001u : 0x00000001u) << i;
            }
        }
        P.ncdf[t] = make_uint4(__float_as_uint(dist), aff, closest, 0u);
    }
}

// Collider pose as glam's Pose3 (rotation quaternion, translation).
__device__ __forceinline__ v3 pose_apply(const DevCollider& c, v3 p) {
    return qrot(quat{c.rot[0], c.rot[1], c.rot[2], c.rot[3]}, p) + mk(c.tra[0], c.tra[1], c.tra[2]);
}

// rigid_particle_update.rs:9-31 gpu_transform_sample_points: world position
// of every rigid particle from its collider's pose at the start of the step.
__global__ void __launch_bounds__(256) k_rigid_transform(DevPtrs P) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.nrp; i += gridDim.x * blockDim.x) {
        const float4 l = P.rp_local[i];
        const DevCollider& c = P.colliders[__float_as_uint(l.w) >> kRigidTriBits];
        const v3 w = pose_apply(c, mk(l.x, l.y, l.z));
        P.rp_world[i] = make_float4(w.x, w.y, w.z, l.w);
    }
}

// solver/p2g_cdf.rs:52-259 gpu_p2g_cdf: one CTA of 64 threads (one per node)
// per active block with rigid entries.  Chunks of 64 listed rigid particles
// are staged in shared memory: their triangle in world space (the local
// vertices times the collider pose, rigid_particle_update.rs:33-54), their
// associated cell round(x / dx) - 1 and collider.  A node within the 3-cell
// range of an entry projects on its triangle; a projection inside the face
// sets the collider's affinity bit (and the sign bit for a node behind the
// face).  The reference keeps the first strictly closer entry in list order;
// the list order here comes from atomics, so the rigid candidates reduce to
// the lowest (distance, collider) pair, which is what the reference's
// ascending-id order gives, and only a strictly closer one replaces the
// analytic colliders' result.
__global__ void __launch_bounds__(64) k_p2g_cdf(DevPtrs P) {
    // per staged entry: its triangle's vertices a, b, c, the face normal
    // n = (b - a) x (c - a) with |n|, and the three edge normals (edge x n);
    // a node's test then needs only differences and dot products, with the
    // same operations (and roundings) as forming them per node
    __shared__ float4 sa[64], sb[64], sc[64], sn[64], seab[64], sebc[64], seac[64];
    __shared__ int4 sassoc[64];  // associated cell, collider
    const float dx = P.params->dx;
    const uint32_t nb = __ldcg(&P.counters->num_blocks);
    const uint32_t tid = threadIdx.x;
    for (uint32_t b = blockIdx.x; b < nb; b += gridDim.x) {
        const uint32_t num = P.rp_count[b];
        if (num == 0) continue;
        const uint32_t first = P.rp_first[b];
        int4 vid = P.bvid[b];
        // batched scenes: scene-local cells, and the scene's colliders numbered
        // from its first one (the affinity bits and closest-collider index of
        // the node field are per scene, as for the analytic colliders)
        uint32_t col0 = 0u;
        if (P.params->scene_blocks) {
            const uint32_t sid = scene_of_block(*P.params, vid);
            col0 = sid != NONE ? P.scene_cols[sid].x : 0u;
            const int3 o = scene_base_of_block(*P.params, vid);
            vid.x -= o.x; vid.y -= o.y; vid.z -= o.z;
        }
        const int cx = vid.x * 4 + (int)(tid & 3u), cy = vid.y * 4 + (int)((tid >> 2) & 3u),
                  cz = vid.z * 4 + (int)(tid >> 4);
        const v3 cell_pos = mk((float)cx, (float)cy, (float)cz) * dx;
        const uint4 nc = P.ncdf[b * 64u + tid];
        uint32_t aff = nc.y;
        float rbest = MAX_FLT;
        uint32_t rcol = NONE;
        for (uint32_t chunk = 0; chunk < num; chunk += 64u) {
            __syncthreads();
            if (chunk + tid < num) {
                const uint32_t id = P.rp_sorted[first + chunk + tid];
                const float4 w = P.rp_world[id];
                const uint32_t word = __float_as_uint(w.w);
                const uint32_t col = word >> kRigidTriBits;
                const DevCollider& c = P.colliders[col];
                const DevTri& t = P.tris[word & kRigidTriMask];
                const v3 a = pose_apply(c, mk(t.v[0][0], t.v[0][1], t.v[0][2]));
                const v3 bb = pose_apply(c, mk(t.v[1][0], t.v[1][1], t.v[1][2]));
                const v3 cc = pose_apply(c, mk(t.v[2][0], t.v[2][1], t.v[2][2]));
                const v3 ab = bb - a, acv = cc - a, bc = cc - bb;
                const v3 n = cross(ab, acv);
                const float nl = length(n);
                const v3 eab = cross(ab, n), ebc = cross(bc, n), eac = cross(acv, n);
                sa[tid] = make_float4(a.x, a.y, a.z, 0.f);
                sb[tid] = make_float4(bb.x, bb.y, bb.z, 0.f);
                sc[tid] = make_float4(cc.x, cc.y, cc.z, 0.f);
                sn[tid] = make_float4(n.x, n.y, n.z, nl);
                seab[tid] = make_float4(eab.x, eab.y, eab.z, 0.f);
                sebc[tid] = make_float4(ebc.x, ebc.y, ebc.z, 0.f);
                seac[tid] = make_float4(eac.x, eac.y, eac.z, 0.f);
                const v3 ac = assoc_cell_of(dx, mk(w.x, w.y, w.z));
                // a degenerate triangle (|n| = 0) projects on no node: out of every range
                sassoc[tid] = nl != 0.f ? make_int4(f2i_sat(ac.x), f2i_sat(ac.y), f2i_sat(ac.z), (int)(col - col0))
                                        : make_int4(INT32_MIN, INT32_MIN, INT32_MIN, 0);
            }
            __syncthreads();
            const uint32_t len = min(64u, num - chunk);
            for (uint32_t p = 0; p < len; ++p) {
                const int4 as = sassoc[p];
                const unsigned sx = (unsigned)cx - (unsigned)as.x, sy = (unsigned)cy - (unsigned)as.y,
                               sz = (unsigned)cz - (unsigned)as.z;
                if (sx > 2u || sy > 2u || sz > 2u) continue;
                const float4 fa = sa[p];
                const v3 ap = cell_pos - mk(fa.x, fa.y, fa.z);
                const float4 e0 = seab[p];
                if (!(dot(mk(e0.x, e0.y, e0.z), ap) <= 0.f)) continue;
                const float4 fb = sb[p], e1 = sebc[p];
                if (!(dot(mk(e1.x, e1.y, e1.z), cell_pos - mk(fb.x, fb.y, fb.z)) <= 0.f)) continue;
                const float4 fc = sc[p], e2 = seac[p];
                if (!(dot(mk(e2.x, e2.y, e2.z), cell_pos - mk(fc.x, fc.y, fc.z)) >= 0.f)) continue;
                const float4 fn = sn[p];
                const float sd = dot(mk(fn.x, fn.y, fn.z), ap) / fn.w;
                const float d = fabsf(sd);
                const uint32_t col = (uint32_t)as.w;
                aff |= (sd < 0.f ? 0x00010001u : 0x00000001u) << col;
                if (d < rbest || (d == rbest && col < rcol)) {
                    rbest = d;
                    rcol = col;
                }
            }
        }
        float dist = __uint_as_float(nc.x);
        uint32_t closest = nc.z;
        if (rbest < dist) {
            dist = rbest;
            closest = rcol;
        }
        P.ncdf[b * 64u + tid] = make_uint4(__float_as_uint(dist), aff, closest, 0u);
    }
}

// solver/g2p_cdf.rs:150-290: per primary particle, its affinity (the node
// bits; sign bits remembered from the previous step, or for a new affinity
// the sign of the weighted node distances) and an MLS fit distance = n . dpt
// + d over the nodes sharing an affinity with it (normal = n / |n|, signed
// distance = d); a singular fit (determinant <= 1e-8) zeroes the record.
// One CTA per primary block, the 6x6x6 node field in shared memory.
__global__ void __launch_bounds__(128) k_g2p_cdf(DevPtrs P) {
    __shared__ uint4 halo[216];
    const Params prm = *P.params;
    const float dx = prm.dx;
    const uint32_t nbp = min(__ldcg(&P.counters->num_primary), __ldcg(&P.counters->num_blocks));
    for (uint32_t b = blockIdx.x; b < nbp; b += gridDim.x) {
        uint32_t any = 0u;
        for (uint32_t t = threadIdx.x; t < 216u; t += blockDim.x) {
            const uint32_t tx = t % 6u, ty = (t / 6u) % 6u, tz = t / 36u;
            const uint32_t ox = tx >= 4u, oy = ty >= 4u, oz = tz >= 4u;
            const uint32_t oct = ox * 4u + oy * 2u + oz;
            const uint32_t blk = oct == 0 ? b : P.nbh[b * NUM_NBH + oct - 1u];
            halo[t] = blk == NONE ? make_uint4(__float_as_uint(MAX_FLT), 0u, NONE, 0u)
                                  : P.ncdf[blk * 64u + (tx - 4u * ox) + 4u * (ty - 4u * oy) + 16u * (tz - 4u * oz)];
            any |= halo[t].y;
        }
        // a halo without affinity bits gives every particle of the block the zero record
        const bool block_aff = __syncthreads_or((int)(any & 0x0000FFFFu)) != 0;
        const uint32_t first = P.first[b], np = P.nprim[b];
        for (uint32_t k = threadIdx.x; k < np; k += blockDim.x) {
            const uint32_t pid = P.sorted[first + k];
            float4* rec = &P.pcdf[3u * pid];
            const uint32_t prev = __float_as_uint(rec[1].w);
            if (!block_aff) {
                if (prev != 0u) {
                    rec[0] = make_float4(0.f, 0.f, 0.f, 0.f);
                    rec[1] = make_float4(0.f, 0.f, 0.f, __uint_as_float(0u));
                }
                continue;
            }
            const float4 xm = reinterpret_cast<const float4*>(&P.kin[pid])[0];
            const v3 pt = mk(xm.x, xm.y, xm.z);
            const v3 ref = assoc_cell_of(dx, pt) * dx - pt;
            const v3 w0 = kernel_eval_all(-ref.x / dx), w1 = kernel_eval_all(-ref.y / dx),
                     w2 = kernel_eval_all(-ref.z / dx);
            const CellInfo ci = cell_info(dx, pt);
            const uint32_t packed = ci.ax + 6u * ci.ay + 36u * ci.az;
            // the union of the 27 nodes' affinity bits; without any, no node
            // enters the fit, which is then singular: the record is zeroed
            // (and a record whose previous affinity word is 0 is zero already)
            uint32_t pa = 0u;
            for (int i = 0; i < 27; ++i) {
                int sx, sy, sz;
                nbh_shift(i, sx, sy, sz);
                pa |= halo[packed + (uint32_t)(sx + 6 * sy + 36 * sz)].y;
            }
            pa &= 0x0000FFFFu;
            if (pa == 0u) {
                if (prev != 0u) {
                    rec[0] = make_float4(0.f, 0.f, 0.f, 0.f);
                    rec[1] = make_float4(0.f, 0.f, 0.f, __uint_as_float(0u));
                }
                continue;
            }
            // The fit's moment matrix is a weighted sum of p p^T (positive
            // semi-definite), so its determinant is at most the product of its
            // diagonal (Hadamard's inequality); the float evaluation of the
            // determinant stays within a relative 1e-3 above that product, so
            // a product at or below 1e-8 / 1.01 leaves the fit singular and
            // the record zero (whatever the signs below).  The diagonal is
            // summed as in the full pass, over the same nodes (affinity bits).
            {
                float dg[4] = {0.f, 0.f, 0.f, 0.f};
                for (int i = 0; i < 27; ++i) {
                    int sx, sy, sz;
                    nbh_shift(i, sx, sy, sz);
                    const uint4 nd = halo[packed + (uint32_t)(sx + 6 * sy + 36 * sz)];
                    if (!(nd.y & pa & 0x0000FFFFu)) continue;
                    const v3 dpt = ref + mk((float)sx, (float)sy, (float)sz) * dx;
                    const float weight = vget(w0, sx) * vget(w1, sy) * vget(w2, sz);
                    dg[0] += dpt.x * dpt.x * weight;
                    dg[1] += dpt.y * dpt.y * weight;
                    dg[2] += dpt.z * dpt.z * weight;
                    dg[3] += 1.0f * 1.0f * weight;
                }
                if (dg[0] * dg[1] * dg[2] * dg[3] * 1.01f <= 1.0e-8f) {
                    if (prev != 0u) {
                        rec[0] = make_float4(0.f, 0.f, 0.f, 0.f);
                        rec[1] = make_float4(0.f, 0.f, 0.f, __uint_as_float(0u));
                    }
                    continue;
                }
            }
            // signs: kept for every collider of the previous affinity (with or
            // without a node carrying it now); for a new affinity, the sign of
            // the weighted distances of the nodes carrying that collider's
            // bit, summed in stencil order (a node without the bit adds zero)
            pa |= prev & ((prev & 0x0000FFFFu) << 16);
            for (uint32_t rem = pa & ~prev & 0x0000FFFFu; rem != 0u; rem &= rem - 1u) {
                const uint32_t bit = rem & (0u - rem);
                float sum = 0.f;
                for (int i = 0; i < 27; ++i) {
                    int sx, sy, sz;
                    nbh_shift(i, sx, sy, sz);
                    const uint4 nd = halo[packed + (uint32_t)(sx + 6 * sy + 36 * sz)];
                    if (!(nd.y & bit)) continue;
                    const float weight = vget(w0, sx) * vget(w1, sy) * vget(w2, sz);
                    const float sign = ((nd.y >> 16) & bit) ? -1.0f : 1.0f;
                    sum += weight * sign * __uint_as_float(nd.x);
                }
                if (sum < 0.f) pa |= bit << 16;
            }
            float q[4][4], u[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int c = 0; c < 4; ++c) q[r][c] = 0.f;
            for (int i = 0; i < 27; ++i) {
                int sx, sy, sz;
                nbh_shift(i, sx, sy, sz);
                const uint4 nd = halo[packed + (uint32_t)(sx + 6 * sy + 36 * sz)];
                const v3 dpt = ref + mk((float)sx, (float)sy, (float)sz) * dx;
                const float weight = vget(w0, sx) * vget(w1, sy) * vget(w2, sz);
                const uint32_t combined = nd.y & pa & 0x0000FFFFu;
                const uint32_t sdiff = ((nd.y >> 16) ^ (pa >> 16)) & combined;
                const float pv[4] = {dpt.x, dpt.y, dpt.z, 1.0f};
                if (combined != 0u) {
                    const float ndist = __uint_as_float(nd.x);
                    const float dd = sdiff == 0u ? ndist : -ndist;
#pragma unroll
                    for (int r = 0; r < 4; ++r)
#pragma unroll
                        for (int c = 0; c < 4; ++c) q[r][c] += pv[r] * pv[c] * weight;
#pragma unroll
                    for (int r = 0; r < 4; ++r) u[r] += pv[r] * (weight * dd);
                }
            }
            float qi[4][4];
            const float dt4 = inv4(q, qi);
            if (dt4 > 1.0e-8f) {
                float r4[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) r4[i] = qi[i][0] * u[0] + qi[i][1] * u[1] + qi[i][2] * u[2] + qi[i][3] * u[3];
                const v3 nv = mk(r4[0], r4[1], r4[2]);
                const float len = length(nv);
                const v3 n = len > 1.0e-6f ? nv / len : splat(0.f);
                rec[0] = make_float4(n.x, n.y, n.z, r4[3]);
                rec[1] = make_float4(0.f, 0.f, 0.f, __uint_as_float(pa));
            } else {
                rec[0] = make_float4(0.f, 0.f, 0.f, 0.f);
                rec[1] = make_float4(0.f, 0.f, 0.f, __uint_as_float(0u));
            }
        }
        __syncthreads();
    }
}

}  // namespace

void launch_grid_update_cdf(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s) {
    k_grid_update_cdf<<<c.sm_count * 8, 256, 0, s>>>(P);
}

void launch_g2p_cdf(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s) {
    k_g2p_cdf<<<c.sm_count * 4, 128, 0, s>>>(P);
}

void launch_rigid_transform(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s) {
    k_rigid_transform<<<c.sm_count * 4, 256, 0, s>>>(P);
}

void launch_p2g_cdf(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s) {
    k_p2g_cdf<<<c.sm_count * 16, 64, 0, s>>>(P);
}

void launch_timestep_bound(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s) {
    k_timestep_bound<<<c.sm_count * 4, 256, 0, s>>>(P);
}

void launch_p2g_gather(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s) {
    k_p2g_gather<<<c.sm_count * 16, 64, 0, s>>>(P);
}

}  // namespace exact
}  // namespace nxm
