// Deterministic-mode transfers, built with --fmad=false: the reference's
// atomic-free, gather-form P2G (solver/p2g.rs:64-351, USE_CPIC = false) with
// its chunking, z-slab culling and summation order, plus the grid update and
// fused G2P + particle update of nxm_transfer.inc.cuh.  Given the canonical
// sort order these reproduce the CPU oracle's f32 arithmetic operation by
// operation (up to the last bits of logf/expf/sinf).
#define NXM_NS exact
#define NXM_FAST false
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
        v3 acc_mv = splat(0.f);
        float acc_mass = 0.f;
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
                    acc_mv = acc_mv + vel_contribution;
                    acc_mass += mass_contribution;
                }
            }
        }
        P.nodes[b * 64u + tid] = make_float4(acc_mv.x, acc_mv.y, acc_mv.z, acc_mass);
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

}  // namespace

void launch_timestep_bound(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s) {
    k_timestep_bound<<<c.sm_count * 4, 256, 0, s>>>(P);
}

void launch_p2g_gather(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s) {
    k_p2g_gather<<<c.sm_count * 16, 64, 0, s>>>(P);
}

}  // namespace exact
}  // namespace nxm
