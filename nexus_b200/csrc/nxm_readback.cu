// Render data of the particles and of the CPIC rigid particles, headless
// (src_mpm_shaders/solver/prep_readback.rs, 3D): per particle a color for the
// render mode, the deformation diag(2 r) * clamp(F, -4, 4) and the position,
// written in particle-id order either as ReadbackData records (color, 4x4
// deformation, position: 96 bytes) or as the three arrays a renderer's
// instance buffers take.  Built with --fmad=false, like the oracle.
//
// One thread per storage slot: the particle records are read where they lie
// (block order in the fast mode) and the result goes to the particle's id.
#include "nxm_device.cuh"
#include "nxm_kernels.h"

namespace nxm {
namespace {

// compute_color (prep_readback.rs:176-237) and compute_deformation (:111-123).
__device__ __forceinline__ void render_particle(const RenderSrc& in, uint32_t slot, uint32_t& id, float4& color,
                                                m3& deform, v3& pos) {
    id = in.pid ? in.pid[slot] : slot;
    const float4* kr = reinterpret_cast<const float4*>(&in.kin[slot]);
    const float4 xm = kr[0], vf = kr[1];
    const float4* dr = reinterpret_cast<const float4*>(&in.def[slot]);
    const float4 f0 = dr[0], f1 = dr[1], f2 = dr[2];
    const float4 props = in.pcdf[3u * id + 2u];  // boundary friction, init radius, phase, group id
    const m3 F = mkm(mk(f0.x, f0.y, f0.z), mk(f1.x, f1.y, f1.z), mk(f2.x, f2.y, f2.z));
    pos = mk(xm.x, xm.y, xm.z);
    const uint32_t ng = in.num_groups ? in.num_groups : 1u;
    const float4 base = in.palette[__float_as_uint(props.w) % ng];
    color = base;
    switch (in.mode) {
        case RENDER_VOLUME: {
            const Svd d = svd3(F);
            const v3 c = (splat(1.0f) - d.s) / 0.005f + splat(0.2f);
            color = make_float4(c.x, c.y, c.z, base.w);
            break;
        }
        case RENDER_VELOCITY: {
            const v3 c = vabs(mk(vf.x, vf.y, vf.z)) * in.dt * 100.0f + splat(0.2f);
            color = make_float4(c.x, c.y, c.z, base.w);
            break;
        }
        case RENDER_PHASE:
            color = make_float4(0.0f, 0.4f * props.z, 0.4f * (1.0f - props.z), base.w);
            break;
        case RENDER_CDF_NORMALS: {
            const float4 c0 = in.pcdf[3u * id];
            if (c0.x == 0.0f && c0.y == 0.0f && c0.z == 0.0f) {
                color = make_float4(0.0f, 0.0f, 0.0f, base.w);
            } else {
                const v3 n = (mk(c0.x, c0.y, c0.z) + splat(1.0f)) * 0.5f;
                color = make_float4(n.x, n.y, n.z, base.w);
            }
            break;
        }
        case RENDER_CDF_DISTANCES: {
            const float d = in.pcdf[3u * id].w / (in.dx * 1.5f);
            color = d > 0.0f ? make_float4(0.0f, fabsf(d), 0.0f, base.w) : make_float4(fabsf(d), 0.0f, 0.0f, base.w);
            break;
        }
        case RENDER_CDF_SIGNS: {
            const uint32_t a = __float_as_uint(in.pcdf[3u * id + 1u].w);
            const uint32_t both = (a >> 16) & (a & 0x0000FFFFu);
            color = a == 0u ? make_float4(0.0f, 0.0f, 0.0f, base.w)
                            : (both == 0u ? make_float4(0.0f, 1.0f, 0.0f, base.w)
                                          : make_float4(1.0f, 0.0f, 0.0f, base.w));
            break;
        }
        default:
            break;
    }
    if (!(__float_as_uint(vf.w) & PFLAG_ENABLED)) color = make_float4(1.0f, 0.0f, 0.0f, 1.0f);  // failed
    const m3 cl = mkm(vclamp(F.c0, -4.0f, 4.0f), vclamp(F.c1, -4.0f, 4.0f), vclamp(F.c2, -4.0f, 4.0f));
    deform = diag(splat(props.y * 2.0f)) * cl;
}

// One ReadbackData record: color, deformation as Mat4::from_mat3 (columns),
// position, padding.
__device__ __forceinline__ void store_record(float4* o, float4 color, const m3& d, v3 pos) {
    o[0] = color;
    o[1] = make_float4(d.c0.x, d.c0.y, d.c0.z, 0.0f);
    o[2] = make_float4(d.c1.x, d.c1.y, d.c1.z, 0.0f);
    o[3] = make_float4(d.c2.x, d.c2.y, d.c2.z, 0.0f);
    o[4] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    o[5] = make_float4(pos.x, pos.y, pos.z, 0.0f);
}

// prep_readback.rs:241-295 gpu_prep_readback.
__global__ void __launch_bounds__(256) k_prep_readback(RenderSrc in, float4* __restrict__ out) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < in.n; t += gridDim.x * blockDim.x) {
        uint32_t id;
        float4 color;
        m3 d;
        v3 pos;
        render_particle(in, t, id, color, d, pos);
        store_record(out + 6u * (size_t)id, color, d, pos);
    }
}

// prep_readback.rs:300-357 gpu_mpm_prep_render: positions (3 floats),
// deformations (9, column-major 3x3) and colors (4) per particle.
__global__ void __launch_bounds__(256) k_prep_render(RenderSrc in, float* __restrict__ positions,
                                                     float* __restrict__ deformations, float* __restrict__ colors) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < in.n; t += gridDim.x * blockDim.x) {
        uint32_t id;
        float4 color;
        m3 d;
        v3 pos;
        render_particle(in, t, id, color, d, pos);
        float* p = positions + 3u * (size_t)id;
        p[0] = pos.x; p[1] = pos.y; p[2] = pos.z;
        float* m = deformations + 9u * (size_t)id;
        m[0] = d.c0.x; m[1] = d.c0.y; m[2] = d.c0.z;
        m[3] = d.c1.x; m[4] = d.c1.y; m[5] = d.c1.z;
        m[6] = d.c2.x; m[7] = d.c2.y; m[8] = d.c2.z;
        reinterpret_cast<float4*>(colors)[id] = color;
    }
}

// prep_readback.rs:420-469 gpu_prep_readback_rigid: base color (per rigid
// particle, or the palette cycled over them), deformation diag(0.4 dx),
// world position as of the last step's start.
__global__ void __launch_bounds__(256) k_prep_readback_rigid(const float4* __restrict__ world, uint32_t nrp,
                                                             const float4* __restrict__ colors,
                                                             const float4* __restrict__ palette, uint32_t num_groups,
                                                             float dx, float4* __restrict__ out) {
    const float scale = dx * 0.4f;
    const uint32_t ng = num_groups ? num_groups : 1u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nrp; i += gridDim.x * blockDim.x) {
        const float4 w = world[i];
        store_record(out + 6u * (size_t)i, colors ? colors[i] : palette[i % ng], diag(splat(scale)), mk(w.x, w.y, w.z));
    }
}

int grid_of(const RenderSrc& in, uint32_t n) {
    const uint32_t want = (n + 255u) / 256u;
    const uint32_t cap = (uint32_t)in.sm_count * 8u;
    return (int)(want < 1u ? 1u : (want > cap ? cap : want));
}

}  // namespace

void launch_prep_readback(const RenderSrc& in, float4* out, cudaStream_t s) {
    k_prep_readback<<<grid_of(in, in.n), 256, 0, s>>>(in, out);
}

void launch_prep_render(const RenderSrc& in, float* positions, float* deformations, float* colors, cudaStream_t s) {
    k_prep_render<<<grid_of(in, in.n), 256, 0, s>>>(in, positions, deformations, colors);
}

void launch_prep_readback_rigid(const RenderSrc& in, const float4* world, uint32_t nrp, const float4* colors,
                                float4* out, cudaStream_t s) {
    k_prep_readback_rigid<<<grid_of(in, nrp), 256, 0, s>>>(world, nrp, colors, in.palette, in.num_groups, in.dx, out);
}

}  // namespace nxm
