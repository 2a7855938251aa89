// Device-side types and math of the nexus_mpm MLS-MPM step for sm_100a.
//
// Arithmetic follows the reference shaders operation by operation (glam's
// column-major Mat3, left-to-right accumulation) so that a build with
// --fmad=false reproduces the reference's f32 rounding; the fast build lets
// the compiler contract multiply-adds.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "nxm_layout.h"

namespace nxm {

// ---------------------------------------------------------------------------
// Small vector / matrix helpers (glam order).
// ---------------------------------------------------------------------------

struct v3 {
    float x, y, z;
};
struct m3 {
    v3 c0, c1, c2;  // columns
};

__device__ __forceinline__ v3 mk(float x, float y, float z) { return v3{x, y, z}; }
__device__ __forceinline__ v3 operator+(v3 a, v3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ v3 operator-(v3 a, v3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ v3 operator-(v3 a) { return mk(-a.x, -a.y, -a.z); }
__device__ __forceinline__ v3 operator*(v3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ v3 operator/(v3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ v3 cross(v3 a, v3 b) {
    return mk(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
__device__ __forceinline__ float length(v3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ v3 vabs(v3 a) { return mk(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
__device__ __forceinline__ float vget(v3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
__device__ __forceinline__ v3 splat(float s) { return mk(s, s, s); }
// glam Vec3::clamp = max(min).min(max) with NaN-ignoring f32::max / f32::min.
__device__ __forceinline__ v3 vclamp(v3 a, float lo, float hi) {
    return mk(fminf(fmaxf(a.x, lo), hi), fminf(fmaxf(a.y, lo), hi), fminf(fmaxf(a.z, lo), hi));
}
// Rust f32::clamp: NaN-preserving comparison chain.
__device__ __forceinline__ float rclamp(float a, float lo, float hi) { return a < lo ? lo : (a > hi ? hi : a); }

__device__ __forceinline__ m3 mkm(v3 a, v3 b, v3 c) { return m3{a, b, c}; }
__device__ __forceinline__ m3 mzero() { return mkm(splat(0.f), splat(0.f), splat(0.f)); }
__device__ __forceinline__ m3 mident() { return mkm(mk(1, 0, 0), mk(0, 1, 0), mk(0, 0, 1)); }
__device__ __forceinline__ v3 operator*(const m3& m, v3 v) {
    v3 r = m.c0 * v.x;
    r = r + m.c1 * v.y;
    r = r + m.c2 * v.z;
    return r;
}
__device__ __forceinline__ m3 operator*(const m3& a, const m3& b) { return mkm(a * b.c0, a * b.c1, a * b.c2); }
__device__ __forceinline__ m3 operator+(const m3& a, const m3& b) { return mkm(a.c0 + b.c0, a.c1 + b.c1, a.c2 + b.c2); }
__device__ __forceinline__ m3 operator-(const m3& a, const m3& b) { return mkm(a.c0 - b.c0, a.c1 - b.c1, a.c2 - b.c2); }
__device__ __forceinline__ m3 operator*(const m3& a, float s) { return mkm(a.c0 * s, a.c1 * s, a.c2 * s); }
__device__ __forceinline__ m3 transpose(const m3& a) {
    return mkm(mk(a.c0.x, a.c1.x, a.c2.x), mk(a.c0.y, a.c1.y, a.c2.y), mk(a.c0.z, a.c1.z, a.c2.z));
}
__device__ __forceinline__ float det(const m3& a) { return dot(a.c2, cross(a.c0, a.c1)); }
__device__ __forceinline__ m3 diag(v3 d) { return mkm(mk(d.x, 0, 0), mk(0, d.y, 0), mk(0, 0, d.z)); }
__device__ __forceinline__ float trace(const m3& a) { return a.c0.x + a.c1.y + a.c2.z; }
__device__ __forceinline__ m3 outer(v3 a, v3 b) { return mkm(a * b.x, a * b.y, a * b.z); }

struct quat {
    float x, y, z, w;
};
// glam Quat::mul_vec3.
__device__ __forceinline__ v3 qrot(quat q, v3 v) {
    v3 b = mk(q.x, q.y, q.z);
    float b2 = dot(b, b);
    v3 r = v * (q.w * q.w - b2);
    r = r + b * (dot(v, b) * 2.0f);
    r = r + cross(b, v) * (q.w * 2.0f);
    return r;
}
__device__ __forceinline__ quat qconj(quat q) { return quat{-q.x, -q.y, -q.z, q.w}; }

// ---------------------------------------------------------------------------
// Sparse-grid keys (src_mpm_shaders/grid/grid.rs:101-134, solver/particle.rs:208-225).
// ---------------------------------------------------------------------------

__device__ __forceinline__ uint32_t pack_key(int x, int y, int z) {
    return ((uint32_t)(x + 0x3FF) & 0x7FFu) | (((uint32_t)(y + 0x1FF) & 0x3FFu) << 11) |
           (((uint32_t)(z + 0x3FF) & 0x7FFu) << 21);
}
__device__ __forceinline__ int key_x(uint32_t k) { return (int)(k & 0x7FFu) - 0x3FF; }
__device__ __forceinline__ int key_y(uint32_t k) { return (int)((k >> 11) & 0x3FFu) - 0x1FF; }
__device__ __forceinline__ int key_z(uint32_t k) { return (int)((k >> 21) & 0x7FFu) - 0x3FF; }

__device__ __forceinline__ uint32_t hash_key(uint32_t k) {
    k *= 0xCC9E2D51u;
    k = (k << 15) | (k >> 17);
    k *= 0x1B873593u;
    return k;
}

// Batched scenes: block-key offset of a scene, and scene / offset of a block.
__device__ __forceinline__ int floor_div(int a, int b) {
    const int q = a / b;
    return (a % b != 0 && (a < 0)) ? q - 1 : q;  // b > 0
}
__device__ __forceinline__ int3 scene_base_of(const Params& p, uint32_t sid) {
    if (p.scene_blocks == 0) return make_int3(0, 0, 0);
    const int S = (int)p.scene_blocks;
    const int cx = (int)(sid % p.scene_cells[0]) + p.scene_cmin[0];
    const int cy = (int)((sid / p.scene_cells[0]) % p.scene_cells[1]) + p.scene_cmin[1];
    const int cz = (int)(sid / (p.scene_cells[0] * p.scene_cells[1])) + p.scene_cmin[2];
    return make_int3(cx * S, cy * S, cz * S);
}
__device__ __forceinline__ int3 scene_base_of_block(const Params& p, int4 vid) {
    if (p.scene_blocks == 0) return make_int3(0, 0, 0);
    const int S = (int)p.scene_blocks, M = p.scene_margin;
    return make_int3(floor_div(vid.x + M, S) * S, floor_div(vid.y + M, S) * S, floor_div(vid.z + M, S) * S);
}
// NONE for a block outside every scene cell (a particle that left its region).
__device__ __forceinline__ uint32_t scene_of_block(const Params& p, int4 vid) {
    const int S = (int)p.scene_blocks, M = p.scene_margin;
    const uint32_t cx = (uint32_t)(floor_div(vid.x + M, S) - p.scene_cmin[0]);
    const uint32_t cy = (uint32_t)(floor_div(vid.y + M, S) - p.scene_cmin[1]);
    const uint32_t cz = (uint32_t)(floor_div(vid.z + M, S) - p.scene_cmin[2]);
    if (cx >= p.scene_cells[0] || cy >= p.scene_cells[1] || cz >= p.scene_cells[2]) return NONE;
    return cx + p.scene_cells[0] * (cy + p.scene_cells[1] * cz);
}

// assoc_cell = round(pt / dx) - 1, with an IEEE division as in the reference.
__device__ __forceinline__ v3 assoc_cell_of(float dx, v3 pt) {
    return mk(roundf(__fdiv_rn(pt.x, dx)) - 1.0f, roundf(__fdiv_rn(pt.y, dx)) - 1.0f,
              roundf(__fdiv_rn(pt.z, dx)) - 1.0f);
}
// float -> int32 conversion truncating toward zero, saturating, NaN -> 0 (Rust `as i32`).
__device__ __forceinline__ int f2i_sat(float f) { return __float2int_rz(f); }

struct CellInfo {
    int bx, by, bz;       // primary block
    uint32_t ax, ay, az;  // associated cell inside the block, in [0, 3]
};

// Block and associated cell from the quotient q = pt / dx, already formed.
__device__ __forceinline__ CellInfo cell_info_scaled(v3 q) {
    const v3 a = mk(roundf(q.x) - 1.0f, roundf(q.y) - 1.0f, roundf(q.z) - 1.0f);
    float fx = floorf(a.x / 4.0f), fy = floorf(a.y / 4.0f), fz = floorf(a.z / 4.0f);
    CellInfo c;
    c.bx = f2i_sat(fx);
    c.by = f2i_sat(fy);
    c.bz = f2i_sat(fz);
    c.ax = (uint32_t)__float2uint_rz(a.x - fx * 4.0f);
    c.ay = (uint32_t)__float2uint_rz(a.y - fy * 4.0f);
    c.az = (uint32_t)__float2uint_rz(a.z - fz * 4.0f);
    return c;
}

__device__ __forceinline__ CellInfo cell_info(float dx, v3 pt) {
    v3 a = assoc_cell_of(dx, pt);
    float fx = floorf(a.x / 4.0f), fy = floorf(a.y / 4.0f), fz = floorf(a.z / 4.0f);
    CellInfo c;
    c.bx = f2i_sat(fx);
    c.by = f2i_sat(fy);
    c.bz = f2i_sat(fz);
    // a - floor(a / 4) * 4 is an exact small integer; negative or NaN -> 0 like `as u32`.
    float dxl = a.x - fx * 4.0f, dyl = a.y - fy * 4.0f, dzl = a.z - fz * 4.0f;
    c.ax = (uint32_t)__float2uint_rz(dxl);
    c.ay = (uint32_t)__float2uint_rz(dyl);
    c.az = (uint32_t)__float2uint_rz(dzl);
    return c;
}

// ---------------------------------------------------------------------------
// Quadratic B-spline (src_mpm_shaders/grid/kernel.rs:118-142).
// ---------------------------------------------------------------------------

__device__ __forceinline__ float kernel_eval(float x) {
    float x_abs = fabsf(x);
    float part1 = 0.75f - x_abs * x_abs;
    float part2 = 0.5f * (1.5f - x_abs) * (1.5f - x_abs);
    float lt05 = x_abs < 0.5f ? 1.0f : 0.0f;
    float lt15 = x_abs < 1.5f ? 1.0f : 0.0f;
    return lt05 * part1 + (1.0f - lt05) * lt15 * part2;
}
__device__ __forceinline__ v3 kernel_eval_all(float x) {
    return mk(0.5f * (1.5f - x) * (1.5f - x), 0.75f - (x - 1.0f) * (x - 1.0f), 0.5f * (x - 0.5f) * (x - 0.5f));
}

// Stencil order of the reference's G2P (kernel.rs:42-70): z in (2,0,1) outer,
// x in (2,0,1), y in (2,0,1) inner.
__device__ __forceinline__ void nbh_shift(int i, int& sx, int& sy, int& sz) {
    const int ord[3] = {2, 0, 1};
    sz = ord[i / 9];
    sx = ord[(i / 3) % 3];
    sy = ord[i % 3];
}

// ---------------------------------------------------------------------------
// 3x3 SVD: one-sided Jacobi (Hestenes) on the columns of F, in float.
// ---------------------------------------------------------------------------

struct Svd {
    m3 u;
    v3 s;
    m3 vt;
};

// One Jacobi rotation of columns p, q; returns |a_p . a_q| / (|a_p| |a_q|)
// before the rotation (0 when the pair is already orthogonal to 1e-6).
__device__ __forceinline__ float jacobi_pair(float (&a)[3][3], float (&v)[3][3], int p, int q) {
    float alpha = a[0][p] * a[0][p] + a[1][p] * a[1][p] + a[2][p] * a[2][p];
    float beta = a[0][q] * a[0][q] + a[1][q] * a[1][q] + a[2][q] * a[2][q];
    float gamma = a[0][p] * a[0][q] + a[1][p] * a[1][q] + a[2][p] * a[2][q];
    if (fabsf(gamma) <= 1.0e-30f || fabsf(gamma) <= 1.0e-6f * sqrtf(alpha * beta)) return 0.0f;
    float zeta = (beta - alpha) / (2.0f * gamma);
    float t = copysignf(1.0f, zeta) / (fabsf(zeta) + sqrtf(1.0f + zeta * zeta));
    float c = rsqrtf(1.0f + t * t);
    float s = c * t;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        float ap = a[r][p], aq = a[r][q];
        a[r][p] = c * ap - s * aq;
        a[r][q] = s * ap + c * aq;
        float vp = v[r][p], vq = v[r][q];
        v[r][p] = c * vp - s * vq;
        v[r][q] = s * vp + c * vq;
    }
    return fabsf(gamma) * rsqrtf(alpha * beta);
}

__device__ __forceinline__ Svd svd3(const m3& f) {
    float a[3][3] = {{f.c0.x, f.c1.x, f.c2.x}, {f.c0.y, f.c1.y, f.c2.y}, {f.c0.z, f.c1.z, f.c2.z}};
    float v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
#pragma unroll 1
    // cyclic sweeps until every column pair is orthogonal to 1e-6 (two or
    // three sweeps for the near-rotation deformation gradients of MPM; at most 10)
    for (int sweep = 0; sweep < 10; ++sweep) {
        float off = jacobi_pair(a, v, 0, 1);
        off = fmaxf(off, jacobi_pair(a, v, 0, 2));
        off = fmaxf(off, jacobi_pair(a, v, 1, 2));
        if (off == 0.0f) break;
    }
    float sig[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) sig[c] = sqrtf(a[0][c] * a[0][c] + a[1][c] * a[1][c] + a[2][c] * a[2][c]);
    // sort decreasing (3-element network), swapping columns of a and v
    auto swapc = [&](int i, int j) {
        float t = sig[i]; sig[i] = sig[j]; sig[j] = t;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            float ta = a[r][i]; a[r][i] = a[r][j]; a[r][j] = ta;
            float tv = v[r][i]; v[r][i] = v[r][j]; v[r][j] = tv;
        }
    };
    if (sig[1] > sig[0]) swapc(0, 1);
    if (sig[2] > sig[0]) swapc(0, 2);
    if (sig[2] > sig[1]) swapc(1, 2);
    float u[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        float inv = sig[c] > 1.0e-30f ? 1.0f / sig[c] : 0.0f;
#pragma unroll
        for (int r = 0; r < 3; ++r) u[r][c] = a[r][c] * inv;
    }
    if (!(sig[1] > 1.0e-30f)) {
        float ux = u[0][0], uy = u[1][0], uz = u[2][0];
        float ox, oy, oz;
        if (fabsf(ux) < 0.9f) { ox = 0; oy = -uz; oz = uy; } else { ox = uz; oy = 0; oz = -ux; }
        float on = sqrtf(ox * ox + oy * oy + oz * oz);
        if (on == 0.0f) { ox = 1; oy = 0; oz = 0; on = 1; }
        u[0][1] = ox / on; u[1][1] = oy / on; u[2][1] = oz / on;
    }
    if (!(sig[2] > 1.0e-30f)) {
        u[0][2] = u[1][0] * u[2][1] - u[2][0] * u[1][1];
        u[1][2] = u[2][0] * u[0][1] - u[0][0] * u[2][1];
        u[2][2] = u[0][0] * u[1][1] - u[1][0] * u[0][1];
    }
    Svd out;
    out.u = mkm(mk(u[0][0], u[1][0], u[2][0]), mk(u[0][1], u[1][1], u[2][1]), mk(u[0][2], u[1][2], u[2][2]));
    out.s = mk(sig[0], sig[1], sig[2]);
    out.vt = mkm(mk(v[0][0], v[0][1], v[0][2]), mk(v[1][0], v[1][1], v[1][2]), mk(v[2][0], v[2][1], v[2][2]));
    return out;
}

// Fast-build SVD: the same Jacobi sweeps with the orthogonality test on
// squares (no square roots), the rotation's division by an approximate
// reciprocal (__fdividef), and the singular values and U columns from one
// reciprocal square root per column.  Agrees with svd3 to a few ulp.
__device__ __forceinline__ bool jacobi_pair_fast(float (&a)[3][3], float (&v)[3][3], int p, int q) {
    const float alpha = a[0][p] * a[0][p] + a[1][p] * a[1][p] + a[2][p] * a[2][p];
    const float beta = a[0][q] * a[0][q] + a[1][q] * a[1][q] + a[2][q] * a[2][q];
    const float gamma = a[0][p] * a[0][q] + a[1][p] * a[1][q] + a[2][p] * a[2][q];
    if (gamma * gamma <= 1.0e-12f * alpha * beta || fabsf(gamma) <= 1.0e-30f) return false;
    const float zeta = __fdividef(beta - alpha, 2.0f * gamma);
    const float t = __fdividef(copysignf(1.0f, zeta), fabsf(zeta) + sqrtf(1.0f + zeta * zeta));
    const float c = rsqrtf(1.0f + t * t);
    const float s = c * t;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        const float ap = a[r][p], aq = a[r][q];
        a[r][p] = c * ap - s * aq;
        a[r][q] = s * ap + c * aq;
        const float vp = v[r][p], vq = v[r][q];
        v[r][p] = c * vp - s * vq;
        v[r][q] = s * vp + c * vq;
    }
    return true;
}

__device__ __forceinline__ Svd svd3_fast(const m3& f) {
    float a[3][3] = {{f.c0.x, f.c1.x, f.c2.x}, {f.c0.y, f.c1.y, f.c2.y}, {f.c0.z, f.c1.z, f.c2.z}};
    float v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
#pragma unroll 1
    for (int sweep = 0; sweep < 10; ++sweep) {
        bool rot = jacobi_pair_fast(a, v, 0, 1);
        rot |= jacobi_pair_fast(a, v, 0, 2);
        rot |= jacobi_pair_fast(a, v, 1, 2);
        if (!rot) break;
    }
    float sig[3], inv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float n2 = a[0][c] * a[0][c] + a[1][c] * a[1][c] + a[2][c] * a[2][c];
        inv[c] = n2 > 1.0e-36f ? rsqrtf(n2) : 0.0f;
        sig[c] = n2 * inv[c];
    }
    auto swapc = [&](int i, int j) {
        float t = sig[i]; sig[i] = sig[j]; sig[j] = t;
        t = inv[i]; inv[i] = inv[j]; inv[j] = t;
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            float ta = a[r][i]; a[r][i] = a[r][j]; a[r][j] = ta;
            float tv = v[r][i]; v[r][i] = v[r][j]; v[r][j] = tv;
        }
    };
    if (sig[1] > sig[0]) swapc(0, 1);
    if (sig[2] > sig[0]) swapc(0, 2);
    if (sig[2] > sig[1]) swapc(1, 2);
    float u[3][3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 3; ++r) u[r][c] = a[r][c] * inv[c];
    if (!(sig[1] > 1.0e-18f)) {
        float ux = u[0][0], uy = u[1][0], uz = u[2][0];
        float ox, oy, oz;
        if (fabsf(ux) < 0.9f) { ox = 0; oy = -uz; oz = uy; } else { ox = uz; oy = 0; oz = -ux; }
        float on = sqrtf(ox * ox + oy * oy + oz * oz);
        if (on == 0.0f) { ox = 1; oy = 0; oz = 0; on = 1; }
        u[0][1] = ox / on; u[1][1] = oy / on; u[2][1] = oz / on;
    }
    if (!(sig[2] > 1.0e-18f)) {
        u[0][2] = u[1][0] * u[2][1] - u[2][0] * u[1][1];
        u[1][2] = u[2][0] * u[0][1] - u[0][0] * u[2][1];
        u[2][2] = u[0][0] * u[1][1] - u[1][0] * u[0][1];
    }
    Svd out;
    out.u = mkm(mk(u[0][0], u[1][0], u[2][0]), mk(u[0][1], u[1][1], u[2][1]), mk(u[0][2], u[1][2], u[2][2]));
    out.s = mk(sig[0], sig[1], sig[2]);
    out.vt = mkm(mk(v[0][0], v[0][1], v[0][2]), mk(v[1][0], v[1][1], v[1][2]), mk(v[2][0], v[2][1], v[2][2]));
    return out;
}

// ---------------------------------------------------------------------------
// Constitutive models (src_mpm_shaders/models/*.rs).
// ---------------------------------------------------------------------------

// linear_elasticity.rs:114-138, given the SVD of F.
__device__ __forceinline__ m3 linear_stress_svd(float lambda, float mu, const m3& F, const Svd& d) {
    float j = d.s.x * d.s.y * d.s.z;
    v3 ms = d.s - splat(1.0f);
    m3 rec = (d.u * diag(ms)) * d.vt;
    float diag_val = lambda * (j - 1.0f) * j;
    m3 res = (rec * transpose(F)) * (2.0f * mu);
    res.c0.x += diag_val;
    res.c1.y += diag_val;
    res.c2.z += diag_val;
    return res;
}
__device__ __forceinline__ m3 linear_stress(float lambda, float mu, const m3& F) {
    return linear_stress_svd(lambda, mu, F, svd3(F));
}

// neo_hookean_elasticity.rs:26-39
__device__ __forceinline__ m3 neo_hookean_stress(float lambda, float mu, const m3& F) {
    float j = fmaxf(det(F), 1.0e-10f);
    float diag_val = lambda * logf(j) - mu;
    m3 st = (F * transpose(F)) * mu;
    st.c0.x += diag_val;
    st.c1.y += diag_val;
    st.c2.z += diag_val;
    return st;
}

// fluid.rs:54-85; p = [bulk_modulus, gamma, viscosity, cfl_coeff, tensile_stiffness]
__device__ __forceinline__ float fluid_pressure(const float* p, float j) {
    j = fmaxf(j, 1.0e-6f);
    if (j <= 1.0f) {
        float ratio = expf(-p[1] * logf(j));
        return p[0] * (ratio - 1.0f);
    }
    return -p[0] * p[4] * (j - 1.0f);
}
__device__ __forceinline__ m3 fluid_stress(const float* p, const m3& F, const m3& strain_rate) {
    float j = fmaxf(det(F), 1.0e-6f);
    float sph = trace(strain_rate) / 3.0f;
    m3 dev = strain_rate;
    dev.c0.x -= sph;
    dev.c1.y -= sph;
    dev.c2.z -= sph;
    m3 st = dev * (2.0f * p[2] * j);
    float diag_val = -fluid_pressure(p, j) * j;
    st.c0.x += diag_val;
    st.c1.y += diag_val;
    st.c2.z += diag_val;
    return st;
}

// drucker_prager.rs:64-67; pl = [ha, hb, hc, hd, lambda, mu, cohesion]
__device__ __forceinline__ float dp_alpha(const float* pl, float q) {
    float angle = pl[0] + (pl[1] * q - pl[3]) * expf(-pl[2] * q);
    float s_angle = sinf(angle);
    return sqrtf(2.0f / 3.0f) * (2.0f * s_angle) / (3.0f - s_angle);
}

// drucker_prager.rs:121-167 and :224-267; state = [pdet, hardening, log_vol_gain].
// `d` receives an SVD of the returned F: the projected F is U diag(sv) V^T,
// so its SVD is known without recomputing it.
__device__ __forceinline__ m3 dp_project_svd(const float* pl, float* state, const m3& F, Svd& d) {
    d = svd3(F);
    if (pl[4] == 0.0f) return F;
    float alpha = dp_alpha(pl, state[1]);
    const float dd = 3.0f;
    v3 strain = mk(logf(d.s.x), logf(d.s.y), logf(d.s.z)) + splat(state[2] / dd);
    float tr = strain.x + strain.y + strain.z;
    v3 dev = strain - splat(tr / dd);
    float shifted = tr - pl[6];
    v3 sv;
    float hard;
    if (shifted > 0.0f || (dev.x == 0.0f && dev.y == 0.0f && dev.z == 0.0f)) {
        sv = splat(expf(pl[6] / dd));
        hard = length(strain);
    } else {
        float dnorm = length(dev);
        float gamma = dnorm + (dd * pl[4] + 2.0f * pl[5]) / (2.0f * pl[5]) * shifted * alpha;
        if (gamma <= 0.0f) return F;  // invalid projection: state and F unchanged
        v3 h = strain - dev * (gamma / dnorm);
        sv = mk(expf(h.x), expf(h.y), expf(h.z));
        hard = gamma;
    }
    float prev_det = d.s.x * d.s.y * d.s.z;
    float new_det = sv.x * sv.y * sv.z;
    float npdet = state[0] * prev_det / new_det;
    float nlvg = state[2] + logf(prev_det) - logf(new_det);
    float nhard = state[1] + hard;
    state[0] = npdet;
    state[1] = nhard;
    state[2] = nlvg;
    d.s = sv;
    return (d.u * diag(sv)) * d.vt;
}
// Fast-build Drucker-Prager projection: dp_project_svd's return map with the
// hardware approximations of log, exp and sin (__logf, __expf, __sinf), and
// the determinants' logarithms taken from the strains (log det = sum of the
// log singular values), so no further logarithm is needed.
// The paths that leave F unchanged return it as U S V^T (equal to rounding),
// so F itself need not stay live across the SVD.
__device__ __forceinline__ m3 dp_project_fast(const float* pl, float* state, const m3& F, Svd& d) {
    d = svd3_fast(F);
    if (pl[4] == 0.0f) return (d.u * diag(d.s)) * d.vt;
    const float q = state[1];
    const float angle = pl[0] + (pl[1] * q - pl[3]) * __expf(-pl[2] * q);
    const float s_angle = __sinf(angle);
    const float alpha = sqrtf(2.0f / 3.0f) * __fdividef(2.0f * s_angle, 3.0f - s_angle);
    const float dd = 3.0f;
    const v3 ls = mk(__logf(d.s.x), __logf(d.s.y), __logf(d.s.z));
    const v3 strain = ls + splat(state[2] / dd);
    const float tr = strain.x + strain.y + strain.z;
    const v3 dev = strain - splat(tr / dd);
    const float shifted = tr - pl[6];
    v3 sv;
    float hard, log_new;
    if (shifted > 0.0f || (dev.x == 0.0f && dev.y == 0.0f && dev.z == 0.0f)) {
        sv = splat(__expf(pl[6] / dd));
        hard = length(strain);
        log_new = pl[6];
    } else {
        const float dnorm = length(dev);
        const float gamma = dnorm + (dd * pl[4] + 2.0f * pl[5]) / (2.0f * pl[5]) * shifted * alpha;
        if (gamma <= 0.0f) return (d.u * diag(d.s)) * d.vt;  // invalid projection: state and F unchanged
        const v3 h = strain - dev * __fdividef(gamma, dnorm);
        sv = mk(__expf(h.x), __expf(h.y), __expf(h.z));
        hard = gamma;
        log_new = h.x + h.y + h.z;
    }
    const float log_prev = ls.x + ls.y + ls.z;
    state[0] = state[0] * __expf(log_prev - log_new);
    state[1] = state[1] + hard;
    state[2] = state[2] + log_prev - log_new;
    d.s = sv;
    return (d.u * diag(sv)) * d.vt;
}

// Fast-build corotated linear stress from the SVD of F: with F = U S V^T,
// U (S - I) V^T F^T = U diag((s - 1) s) U^T, a symmetric product.
__device__ __forceinline__ m3 linear_stress_fast(float lambda, float mu, const Svd& d) {
    const float j = d.s.x * d.s.y * d.s.z;
    const v3 e = mk((d.s.x - 1.0f) * d.s.x, (d.s.y - 1.0f) * d.s.y, (d.s.z - 1.0f) * d.s.z) * (2.0f * mu);
    const m3& U = d.u;
    const v3 u0e = U.c0 * e.x, u1e = U.c1 * e.y, u2e = U.c2 * e.z;
    const float xx = u0e.x * U.c0.x + u1e.x * U.c1.x + u2e.x * U.c2.x;
    const float yy = u0e.y * U.c0.y + u1e.y * U.c1.y + u2e.y * U.c2.y;
    const float zz = u0e.z * U.c0.z + u1e.z * U.c1.z + u2e.z * U.c2.z;
    const float xy = u0e.x * U.c0.y + u1e.x * U.c1.y + u2e.x * U.c2.y;
    const float xz = u0e.x * U.c0.z + u1e.x * U.c1.z + u2e.x * U.c2.z;
    const float yz = u0e.y * U.c0.z + u1e.y * U.c1.z + u2e.y * U.c2.z;
    const float diag_val = lambda * (j - 1.0f) * j;
    return mkm(mk(xx + diag_val, xy, xz), mk(xy, yy + diag_val, yz), mk(xz, yz, zz + diag_val));
}

__device__ __forceinline__ m3 dp_project(const float* pl, float* state, const m3& F) {
    Svd d;
    return dp_project_svd(pl, state, F, d);
}

// snow.rs:452-488; state = [plastic_det]; pl = [critical_compression, critical_stretch, hardening]
__device__ __forceinline__ m3 snow_project(const float* pl, float* state, const m3& F, float* hardening) {
    if (pl[0] <= 0.0f && pl[1] <= 0.0f) {
        *hardening = expf(pl[2] * (1.0f - state[0]));
        return F;
    }
    Svd d = svd3(F);
    float lo = 1.0f - pl[0];
    float hi = 1.0f + pl[1];
    v3 cl = vclamp(d.s, lo, hi);
    float prev_det = d.s.x * d.s.y * d.s.z;
    float new_det = cl.x * cl.y * cl.z;
    float pdet = rclamp(state[0] * prev_det / new_det, 0.1f, 4.0f);
    state[0] = pdet;
    *hardening = expf(pl[2] * (1.0f - pdet));
    return (d.u * diag(cl)) * d.vt;
}

// models/default.rs:208-264.  `w` holds the material's 24 model words; the
// per-particle state words (Drucker-Prager words 0..2, snow word 0) are in `st`
// and updated in place.  kReuseSvd selects the fast build's forms, which
// agree with the reference's to rounding: Drucker-Prager sand on a linear
// backbone takes its stress from the projection's SVD instead of a second SVD
// of the projected F, with the fast SVD, projection and stress above; the
// deterministic build keeps the reference's operation order.
template <bool kReuseSvd>
__device__ __forceinline__ m3 model_update(uint32_t tag, const float* w, float* st, m3& F, const m3& vel_grad) {
    switch (tag) {
    case MODEL_ELASTIC_LINEAR:
        if (kReuseSvd) return linear_stress_fast(w[0], w[1], svd3_fast(F));
        return linear_stress(w[0], w[1], F);
    case MODEL_ELASTIC_NEO_HOOKEAN:
        return neo_hookean_stress(w[0], w[1], F);
    case MODEL_SAND_LINEAR:
        if (kReuseSvd) {
            Svd d;
            F = dp_project_fast(&w[3], st, F, d);
            return linear_stress_fast(w[10], w[11], d);
        } else {
            F = dp_project(&w[3], st, F);
            return linear_stress(w[10], w[11], F);
        }
    case MODEL_SAND_NEO_HOOKEAN:
        if (kReuseSvd) {
            Svd d;
            F = dp_project_fast(&w[3], st, F, d);
        } else {
            F = dp_project(&w[3], st, F);
        }
        return neo_hookean_stress(w[10], w[11], F);
    case MODEL_FLUID: {
        m3 sr = (vel_grad + transpose(vel_grad)) * 0.5f;
        return fluid_stress(&w[0], F, sr);
    }
    case MODEL_SNOW: {
        float hard;
        F = snow_project(&w[1], st, F, &hard);
        return linear_stress(w[4] * hard, w[5] * hard, F);
    }
    default:
        return mzero();
    }
}

// ---------------------------------------------------------------------------
// Colliders (grid_update_collide.rs:30-99, shapes, boundary_condition.rs:165-201).
// ---------------------------------------------------------------------------

struct Proj {
    v3 point;
    bool inside;
};

__device__ __forceinline__ Proj ball_project_local(float radius, v3 pt) {
    float d2 = dot(pt, pt);
    Proj r;
    r.inside = d2 <= radius * radius;
    r.point = pt * (radius / sqrtf(d2));
    return r;
}

// parry3d Aabb::project_local_point, solid = false.
__device__ __forceinline__ Proj cuboid_project_local(v3 half, v3 pt) {
    v3 mins_pt = mk(-half.x, -half.y, -half.z) - pt;
    v3 pt_maxs = pt - half;
    v3 shift = mk(fmaxf(mins_pt.x, 0.f), fmaxf(mins_pt.y, 0.f), fmaxf(mins_pt.z, 0.f)) -
               mk(fmaxf(pt_maxs.x, 0.f), fmaxf(pt_maxs.y, 0.f), fmaxf(pt_maxs.z, 0.f));
    Proj r;
    if (!(shift.x == 0.f && shift.y == 0.f && shift.z == 0.f)) {
        r.inside = false;
        r.point = pt + shift;
        return r;
    }
    float best = -3.0e38f;
    bool is_mins = false;
    int best_id = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float mp = vget(mins_pt, i), pm = vget(pt_maxs, i);
        if (mp < pm) {
            if (pm > best) { best_id = i; is_mins = false; best = pm; }
        } else if (mp > best) {
            best_id = i; is_mins = true; best = mp;
        }
    }
    float val = is_mins ? best : -best;
    v3 s = mk(best_id == 0 ? val : 0.f, best_id == 1 ? val : 0.f, best_id == 2 ? val : 0.f);
    r.inside = true;
    r.point = pt + s;
    return r;
}

__device__ __forceinline__ v3 segment_project_local(v3 a, v3 b, v3 pt) {
    v3 ab = b - a;
    v3 ap = pt - a;
    float ab_ap = dot(ab, ap);
    float sqnab = dot(ab, ab);
    if (ab_ap <= 0.f) return a;
    if (ab_ap >= sqnab) return b;
    float u = ab_ap / sqnab;
    return a + ab * u;
}

__device__ __forceinline__ Proj capsule_project_local(v3 a, v3 b, float radius, v3 pt) {
    v3 pa = segment_project_local(a, b, pt);
    v3 dproj = pt - pa;
    float d = length(dproj);
    Proj r;
    if (d > 0.f) {
        r.inside = d <= radius;
        r.point = pa + dproj * (radius / d);
    } else {
        v3 axis = b - a;
        v3 n = axis / length(axis);
        v3 o = fabsf(n.x) > fabsf(n.y) ? mk(-n.z, 0.f, n.x) : mk(0.f, n.z, -n.y);
        o = o / length(o);
        r.inside = true;
        r.point = pa + o * radius;
    }
    return r;
}

// Closest point on triangle (a, b, c) to p and the feature it lies on
// (Ericson, Real-Time Collision Detection 5.1.5, Voronoi regions): feature 0
// = vertex id 0..2, 1 = edge id 0 = ab, 1 = bc, 2 = ca, 2 = face.  The
// reference projects with parry's triangle query (trimesh.rs:172); both give
// the closest point, the feature numbering follows trimesh.rs:120-140.
struct TriProj {
    v3 point;
    int feature, id;
};
__device__ __forceinline__ TriProj triangle_closest(v3 a, v3 b, v3 c, v3 p) {
    TriProj r;
    const v3 ab = b - a, ac = c - a, ap = p - a;
    const float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.f && d2 <= 0.f) { r.point = a; r.feature = 0; r.id = 0; return r; }
    const v3 bp = p - b;
    const float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.f && d4 <= d3) { r.point = b; r.feature = 0; r.id = 1; return r; }
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
        const float v = d1 / (d1 - d3);
        r.point = a + ab * v; r.feature = 1; r.id = 0; return r;
    }
    const v3 cp = p - c;
    const float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.f && d5 <= d6) { r.point = c; r.feature = 0; r.id = 2; return r; }
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
        const float w = d2 / (d2 - d6);
        r.point = a + ac * w; r.feature = 1; r.id = 2; return r;
    }
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
        const float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        r.point = b + (c - b) * w; r.feature = 1; r.id = 1; return r;
    }
    const float denom = 1.0f / (va + vb + vc);
    const float v = vb * denom, w = vc * denom;
    r.point = a + (ab * v + ac * w);
    r.feature = 2; r.id = 0;
    return r;
}

// parry Aabb::distance_to_local_point(pt, solid = true).
__device__ __forceinline__ float aabb_distance(const DevBvhNode& n, v3 p) {
    const float dx = fmaxf(fmaxf(n.mn[0] - p.x, p.x - n.mx[0]), 0.f);
    const float dy = fmaxf(fmaxf(n.mn[1] - p.y, p.y - n.mx[1]), 0.f);
    const float dz = fmaxf(fmaxf(n.mn[2] - p.z, p.z - n.mx[2]), 0.f);
    return sqrtf(dx * dx + dy * dy + dz * dz);
}

// trimesh.rs:155-207 project_local_point: closest triangle within max_dist
// (the last one found wins ties, "dist <= best"), BVH traversal pruned by box
// distance, then the inside test pn . (p - proj) <= 0 with the pseudo-normal
// of the closest feature.  Returns false when no triangle is within max_dist.
__device__ __forceinline__ bool trimesh_project_local(const DevTri* __restrict__ tris,
                                                      const DevBvhNode* __restrict__ bvh, uint32_t first,
                                                      uint32_t count, v3 pt, float max_dist, Proj& out) {
    float best = max_dist;
    TriProj bp;
    bp.point = pt; bp.feature = 2; bp.id = 0;
    uint32_t best_tri = NONE;
    const uint32_t end = first + count;
    uint32_t curr = first;
    for (uint32_t it = 0; it < count && curr < end; ++it) {
        const DevBvhNode n = bvh[curr];
        if (n.entry & kBvhLeaf) {
            const DevTri& t = tris[n.entry & ~kBvhLeaf];
            const TriProj pr = triangle_closest(mk(t.v[0][0], t.v[0][1], t.v[0][2]), mk(t.v[1][0], t.v[1][1], t.v[1][2]),
                                                mk(t.v[2][0], t.v[2][1], t.v[2][2]), pt);
            const float d = length(pr.point - pt);
            if (d <= best) {
                best = d;
                bp = pr;
                best_tri = n.entry & ~kBvhLeaf;
            }
            curr = n.exit;
        } else {
            curr = aabb_distance(n, pt) <= best ? n.entry : n.exit;
        }
    }
    if (best_tri == NONE) return false;
    const DevTri& t = tris[best_tri];
    const int k = bp.feature == 0 ? bp.id : (bp.feature == 1 ? 3 + bp.id : 6);
    const v3 pn = mk(t.pn[k][0], t.pn[k][1], t.pn[k][2]);
    out.point = bp.point;
    out.inside = dot(pn, pt - bp.point) <= 0.f;
    return true;
}

// CPIC affinity bits (grid/grid.rs:593-645): bit i = affinity to collider
// i, bit 16 + i = on its inside; two sets agree if every common affinity has
// the same sign.
__device__ __forceinline__ bool aff_compatible(uint32_t a, uint32_t b) {
    const uint32_t common = a & b & 0x0000FFFFu;
    return ((a >> 16) & common) == ((b >> 16) & common);
}

// Inverse (into out) and determinant of a 4x4 matrix m[row][col] from its
// 2x2 minors (Laplace expansion along the first two rows).
__device__ __forceinline__ float inv4(const float (&m)[4][4], float (&out)[4][4]) {
    const float s0 = m[0][0] * m[1][1] - m[1][0] * m[0][1];
    const float s1 = m[0][0] * m[1][2] - m[1][0] * m[0][2];
    const float s2 = m[0][0] * m[1][3] - m[1][0] * m[0][3];
    const float s3 = m[0][1] * m[1][2] - m[1][1] * m[0][2];
    const float s4 = m[0][1] * m[1][3] - m[1][1] * m[0][3];
    const float s5 = m[0][2] * m[1][3] - m[1][2] * m[0][3];
    const float c5 = m[2][2] * m[3][3] - m[3][2] * m[2][3];
    const float c4 = m[2][1] * m[3][3] - m[3][1] * m[2][3];
    const float c3 = m[2][1] * m[3][2] - m[3][1] * m[2][2];
    const float c2 = m[2][0] * m[3][3] - m[3][0] * m[2][3];
    const float c1 = m[2][0] * m[3][2] - m[3][0] * m[2][2];
    const float c0 = m[2][0] * m[3][1] - m[3][0] * m[2][1];
    const float det = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
    const float id = 1.0f / det;
    out[0][0] = (m[1][1] * c5 - m[1][2] * c4 + m[1][3] * c3) * id;
    out[0][1] = (-m[0][1] * c5 + m[0][2] * c4 - m[0][3] * c3) * id;
    out[0][2] = (m[3][1] * s5 - m[3][2] * s4 + m[3][3] * s3) * id;
    out[0][3] = (-m[2][1] * s5 + m[2][2] * s4 - m[2][3] * s3) * id;
    out[1][0] = (-m[1][0] * c5 + m[1][2] * c2 - m[1][3] * c1) * id;
    out[1][1] = (m[0][0] * c5 - m[0][2] * c2 + m[0][3] * c1) * id;
    out[1][2] = (-m[3][0] * s5 + m[3][2] * s2 - m[3][3] * s1) * id;
    out[1][3] = (m[2][0] * s5 - m[2][2] * s2 + m[2][3] * s1) * id;
    out[2][0] = (m[1][0] * c4 - m[1][1] * c2 + m[1][3] * c0) * id;
    out[2][1] = (-m[0][0] * c4 + m[0][1] * c2 - m[0][3] * c0) * id;
    out[2][2] = (m[3][0] * s4 - m[3][1] * s2 + m[3][3] * s0) * id;
    out[2][3] = (-m[2][0] * s4 + m[2][1] * s2 - m[2][3] * s0) * id;
    out[3][0] = (-m[1][0] * c3 + m[1][1] * c1 - m[1][2] * c0) * id;
    out[3][1] = (m[0][0] * c3 - m[0][1] * c1 + m[0][2] * c0) * id;
    out[3][2] = (-m[3][0] * s3 + m[3][1] * s1 - m[3][2] * s0) * id;
    out[3][3] = (m[2][0] * s3 - m[2][1] * s1 + m[2][2] * s0) * id;
    return det;
}

__device__ __forceinline__ v3 bc_project(uint32_t ty, float friction, v3 vel, v3 n) {
    if (ty == BC_STICK) return splat(0.f);
    if (ty == BC_SLIP) {
        float nv = dot(vel, n);
        return vel - n * nv;
    }
    if (ty == BC_SEPARATE) {
        float nv = dot(vel, n);
        if (nv < 0.f) {
            v3 t = vel - n * nv;
            float tl = length(t);
            v3 tdir = tl > 1.0e-8f ? t / tl : splat(0.f);
            float pl = tl + friction * nv;
            pl = pl > 0.f ? pl : 0.f;
            return tdir * pl;
        }
        return vel;
    }
    return vel;
}

}  // namespace nxm
