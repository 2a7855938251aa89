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
        const int4 vid = P.bvid[b];
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

}  // namespace

void launch_p2g_gather(const DevPtrs& P, const LaunchCfg& c, cudaStream_t s) {
    k_p2g_gather<<<c.sm_count * 16, 64, 0, s>>>(P);
}

}  // namespace exact
}  // namespace nxm
