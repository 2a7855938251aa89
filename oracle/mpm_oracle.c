/*
 * mpm_oracle.c — TEST INFRASTRUCTURE ONLY.
 *
 * A sequential CPU restatement of one nexus_mpm 3D MLS-MPM step (the `dim3`
 * build of the reference, version 0.5.0).  It is the checker that the CUDA
 * library is compared against and the timed CPU baseline; no product code
 * links, includes or calls it.
 *
 * PARITY UNPINNED: the reference ships no MPM tests, fixtures or golden
 * vectors, and its Rust/SPIR-V code cannot be built here (no Rust toolchain,
 * dependencies not vendored).  This file follows the reference shader source
 * line by line (file:line cited at each function, paths relative to the
 * reference project root); the only pin available is the prefix-sum CPU
 * semantics of src_rbd/utils/prefix_sum.rs:112-136, checked by the tests.
 *
 * Build: compiled twice, with -DREAL=float (the FP32 oracle, following the
 * reference's f32 arithmetic operation by operation, -ffp-contract=off) and
 * -DREAL=double (the FP64 accuracy reference).  Sequential processing in
 * particle-id order gives the canonical form of every result the reference
 * computes with atomics (block header order = first-touch order; particles
 * inside a sort bucket in ascending id).  Blocks and particles are processed
 * in parallel with OpenMP only where each result is independent of the
 * thread schedule (P2G per node, grid update per node, G2P/particle update
 * per particle), so results do not depend on the thread count.
 *
 * Third-party arithmetic at the boundary, restated here:
 *   - glamx 0.3 `MatExt::svd` (models/linear_elasticity.rs:115,
 *     models/drucker_prager.rs:237, models/snow.rs:469): one-sided Jacobi SVD
 *     (Hestenes 1958; Demmel & Veselic 1992) carried out in double precision.
 *   - glam 0.30 Vec3/Mat3/Quat operation order (column-major Mat3,
 *     M*v = c0*v.x + c1*v.y + c2*v.z accumulated left to right).
 *   - parry3d 0.30 Ball/Cuboid `project_point` with solid = false
 *     (src_rbd_shaders/shapes/shape.rs:378-385): closest point on the sphere;
 *     Aabb projection that, for an inside point, moves to the nearest face.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <tgmath.h>
#include <float.h>

#ifndef REAL
#define REAL float
#endif

#define NONE_U32 0xFFFFFFFFu
#define NUM_PRIMARY_BUCKETS 4
#define NUM_EXTRA_BUCKETS 6
#define NUM_BUCKETS 10
#define NUM_NBH 7
#define MAX_FLT ((REAL)1.0e18)
#define MODEL_WORDS 24

/* ------------------------------------------------------------------------ */
/* glam-ordered vector / matrix helpers                                      */
/* ------------------------------------------------------------------------ */

typedef struct { REAL x, y, z; } v3;
typedef struct { v3 c0, c1, c2; } m3; /* columns, glam Mat3 layout */

static inline v3 V(REAL x, REAL y, REAL z) { v3 r = {x, y, z}; return r; }
static inline v3 vadd(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vmul(v3 a, REAL s) { return V(a.x * s, a.y * s, a.z * s); }
static inline v3 vdiv(v3 a, REAL s) { return V(a.x / s, a.y / s, a.z / s); }
static inline v3 vcmul(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline REAL vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 vcross(v3 a, v3 b) {
    return V(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
static inline REAL vlen(v3 a) { return sqrt(vdot(a, a)); }
static inline v3 vneg(v3 a) { return V(-a.x, -a.y, -a.z); }
static inline v3 vabs(v3 a) { return V(fabs(a.x), fabs(a.y), fabs(a.z)); }
/* glam Vec3::clamp(min, max) = self.max(min).min(max) with f32::max/min (NaN-ignoring). */
static inline REAL fmaxr(REAL a, REAL b) { return fmax(a, b); }
static inline REAL fminr(REAL a, REAL b) { return fmin(a, b); }
static inline v3 vclamp(v3 a, REAL lo, REAL hi) {
    return V(fminr(fmaxr(a.x, lo), hi), fminr(fmaxr(a.y, lo), hi), fminr(fmaxr(a.z, lo), hi));
}
/* Rust f32::clamp: NaN-preserving comparison chain. */
static inline REAL rclamp(REAL a, REAL lo, REAL hi) {
    if (a < lo) return lo;
    if (a > hi) return hi;
    return a;
}
static inline REAL vget(v3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
static inline v3 vsplat(REAL s) { return V(s, s, s); }

static inline m3 M(v3 c0, v3 c1, v3 c2) { m3 m = {c0, c1, c2}; return m; }
static inline m3 mzero(void) { return M(V(0, 0, 0), V(0, 0, 0), V(0, 0, 0)); }
static inline m3 mident(void) { return M(V(1, 0, 0), V(0, 1, 0), V(0, 0, 1)); }
static inline v3 mv(m3 m, v3 v) {
    v3 r = vmul(m.c0, v.x);
    r = vadd(r, vmul(m.c1, v.y));
    r = vadd(r, vmul(m.c2, v.z));
    return r;
}
static inline m3 mm(m3 a, m3 b) { return M(mv(a, b.c0), mv(a, b.c1), mv(a, b.c2)); }
static inline m3 madd(m3 a, m3 b) { return M(vadd(a.c0, b.c0), vadd(a.c1, b.c1), vadd(a.c2, b.c2)); }
static inline m3 msub(m3 a, m3 b) { return M(vsub(a.c0, b.c0), vsub(a.c1, b.c1), vsub(a.c2, b.c2)); }
static inline m3 mscale(m3 a, REAL s) { return M(vmul(a.c0, s), vmul(a.c1, s), vmul(a.c2, s)); }
static inline m3 mtr(m3 a) {
    return M(V(a.c0.x, a.c1.x, a.c2.x), V(a.c0.y, a.c1.y, a.c2.y), V(a.c0.z, a.c1.z, a.c2.z));
}
static inline REAL mdet(m3 a) { return vdot(a.c2, vcross(a.c0, a.c1)); }
static inline m3 mdiag(v3 d) { return M(V(d.x, 0, 0), V(0, d.y, 0), V(0, 0, d.z)); }
static inline REAL mtrace(m3 a) { return a.c0.x + a.c1.y + a.c2.z; }
/* g2p.rs:377-381 outer_product(a, b) = from_cols(a*b.x, a*b.y, a*b.z) */
static inline m3 mouter(v3 a, v3 b) { return M(vmul(a, b.x), vmul(a, b.y), vmul(a, b.z)); }

/* Quaternion (x, y, z, w) rotation, glam Quat::mul_vec3. */
typedef struct { REAL x, y, z, w; } quat;
static inline v3 qrot(quat q, v3 v) {
    v3 b = V(q.x, q.y, q.z);
    REAL b2 = vdot(b, b);
    v3 r = vmul(v, q.w * q.w - b2);
    r = vadd(r, vmul(b, vdot(v, b) * (REAL)2.0));
    r = vadd(r, vmul(vcross(b, v), q.w * (REAL)2.0));
    return r;
}
static inline quat qconj(quat q) { quat r = {-q.x, -q.y, -q.z, q.w}; return r; }
static inline quat qmul(quat a, quat b) {
    quat r;
    r.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
    r.x = a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y;
    r.y = a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x;
    r.z = a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w;
    return r;
}

typedef struct { quat rot; v3 tra; } pose3;
static inline v3 pose_apply(pose3 p, v3 v) { return vadd(qrot(p.rot, v), p.tra); }
static inline v3 pose_inv_apply(pose3 p, v3 v) { return qrot(qconj(p.rot), vsub(v, p.tra)); }

/* Rust `as i32` / `as u32` from a float: saturating, NaN -> 0. */
static inline int32_t r_to_i32(REAL f) {
    if (f != f) return 0;
    if (f >= (REAL)2147483647.0) return 2147483647;
    if (f <= (REAL)-2147483648.0) return (-2147483647 - 1);
    return (int32_t)f;
}
static inline uint32_t r_to_u32(REAL f) {
    if (f != f || f <= 0) return 0;
    if (f >= (REAL)4294967295.0) return 0xFFFFFFFFu;
    return (uint32_t)f;
}

static inline uint32_t f2bits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float bits2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

/* ------------------------------------------------------------------------ */
/* Sparse grid keys and hash map: src_mpm_shaders/grid/grid.rs              */
/* ------------------------------------------------------------------------ */

typedef struct { int32_t x, y, z; } i3;

/* grid.rs:101-106 BlockVirtualId::pack (3D): 11/10/11 bits. */
static inline uint32_t pack_key(i3 b) {
    return ((uint32_t)(b.x + 0x3FF) & 0x7FFu) | (((uint32_t)(b.y + 0x1FF) & 0x3FFu) << 11) |
           (((uint32_t)(b.z + 0x3FF) & 0x7FFu) << 21);
}

/* grid.rs:430-436 Murmur3 mix. */
static inline uint32_t hash_key(uint32_t k) {
    k *= 0xCC9E2D51u;
    k = (k << 15) | (k >> 17);
    k *= 0x1B873593u;
    return k;
}

/* grid.rs:121-134 block_associated_to_point: assoc_cell = round(pt/dx) - 1, block = floor(assoc/4). */
static inline v3 assoc_cell_of(REAL dx, v3 pt) {
    return V(round(pt.x / dx) - (REAL)1.0, round(pt.y / dx) - (REAL)1.0, round(pt.z / dx) - (REAL)1.0);
}
static inline i3 block_of_point(REAL dx, v3 pt) {
    v3 a = assoc_cell_of(dx, pt);
    i3 b = {r_to_i32(floor(a.x / (REAL)4.0)), r_to_i32(floor(a.y / (REAL)4.0)),
            r_to_i32(floor(a.z / (REAL)4.0))};
    return b;
}
/* solver/particle.rs:208-225 associated_cell_index_in_block_off_by_one. */
static inline void assoc_in_block(REAL dx, v3 pt, uint32_t out[3]) {
    v3 a = assoc_cell_of(dx, pt);
    v3 blk = V(floor(a.x / (REAL)4.0) * (REAL)4.0, floor(a.y / (REAL)4.0) * (REAL)4.0,
               floor(a.z / (REAL)4.0) * (REAL)4.0);
    v3 d = vsub(a, blk);
    out[0] = r_to_u32(d.x);
    out[1] = r_to_u32(d.y);
    out[2] = r_to_u32(d.z);
}
/* grid.rs:175-212 blocks_associated_to_block: z fastest. */
static const i3 ASSOC_SHIFT[8] = {{0, 0, 0}, {0, 0, 1}, {0, 1, 0}, {0, 1, 1},
                                  {1, 0, 0}, {1, 0, 1}, {1, 1, 0}, {1, 1, 1}};
static inline i3 i3add(i3 a, i3 b) { i3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }

/* grid.rs:318-341 ActiveBlockHeader. */
typedef struct {
    i3 vid;
    uint32_t first_particle;
    uint32_t num_particles;
    uint32_t num_particles_with_extras;
    uint32_t cursors[NUM_BUCKETS];
    uint32_t nbh[NUM_NBH];
    uint32_t first_rigid;     /* CPIC: the block's range of the sorted rigid-particle list */
    uint32_t num_rigid;
} header_t;

/* grid.rs:401-421 Node, with the NodeCdf of grid.rs:367-375 (distance,
 * affinity + sign bits, closest collider). */
typedef struct {
    v3 mv;
    REAL mass;
    v3 mv_incompat;
    REAL mass_incompat;
    REAL cdf_distance;
    uint32_t cdf_aff;
    uint32_t cdf_closest;
} node_t;

/* ------------------------------------------------------------------------ */
/* Quadratic B-spline: src_mpm_shaders/grid/kernel.rs                        */
/* ------------------------------------------------------------------------ */

/* kernel.rs:131-142 branchless eval. */
static inline REAL kernel_eval(REAL x) {
    REAL x_abs = fabs(x);
    REAL part1 = (REAL)0.75 - x_abs * x_abs;
    REAL part2 = (REAL)0.5 * ((REAL)1.5 - x_abs) * ((REAL)1.5 - x_abs);
    REAL lt05 = (x_abs < (REAL)0.5) ? (REAL)1.0 : (REAL)0.0;
    REAL lt15 = (x_abs < (REAL)1.5) ? (REAL)1.0 : (REAL)0.0;
    return lt05 * part1 + ((REAL)1.0 - lt05) * lt15 * part2;
}
/* kernel.rs:118-124 eval_all. */
static inline v3 kernel_eval_all(REAL x) {
    return V((REAL)0.5 * ((REAL)1.5 - x) * ((REAL)1.5 - x), (REAL)0.75 - (x - (REAL)1.0) * (x - (REAL)1.0),
             (REAL)0.5 * (x - (REAL)0.5) * (x - (REAL)0.5));
}
/* kernel.rs:42-80 stencil order and shared-tile offsets. */
static const uint8_t NBH_SHIFTS[27][3] = {
    {2, 2, 2}, {2, 0, 2}, {2, 1, 2}, {0, 2, 2}, {0, 0, 2}, {0, 1, 2}, {1, 2, 2}, {1, 0, 2}, {1, 1, 2},
    {2, 2, 0}, {2, 0, 0}, {2, 1, 0}, {0, 2, 0}, {0, 0, 0}, {0, 1, 0}, {1, 2, 0}, {1, 0, 0}, {1, 1, 0},
    {2, 2, 1}, {2, 0, 1}, {2, 1, 1}, {0, 2, 1}, {0, 0, 1}, {0, 1, 1}, {1, 2, 1}, {1, 0, 1}, {1, 1, 1}};

/* ------------------------------------------------------------------------ */
/* SVD (one-sided Jacobi in double)                                          */
/* ------------------------------------------------------------------------ */

typedef struct { m3 u; v3 s; m3 vt; } svd3;

static svd3 svd(m3 f) {
    /* Hestenes one-sided Jacobi: rotate column pairs of A = F until they are
     * orthogonal, accumulating the rotations in V; then sigma_i = |a_i| and
     * u_i = a_i / sigma_i.  Singular values are returned non-negative and
     * sorted in decreasing order; a zero singular value gets a u column that
     * completes a right-handed orthonormal basis. */
    double a[3][3], v[3][3];
    for (int r = 0; r < 3; ++r) {
        a[r][0] = (double)vget(f.c0, r);
        a[r][1] = (double)vget(f.c1, r);
        a[r][2] = (double)vget(f.c2, r);
    }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) v[r][c] = (r == c) ? 1.0 : 0.0;
    static const int P[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    for (int sweep = 0; sweep < 60; ++sweep) {
        double off = 0.0;
        for (int k = 0; k < 3; ++k) {
            int p = P[k][0], q = P[k][1];
            double alpha = 0, beta = 0, gamma = 0;
            for (int r = 0; r < 3; ++r) {
                alpha += a[r][p] * a[r][p];
                beta += a[r][q] * a[r][q];
                gamma += a[r][p] * a[r][q];
            }
            double scale = sqrt(alpha * beta);
            if (scale == 0.0 || fabs(gamma) <= 1e-300) continue;
            double rel = fabs(gamma) / scale;
            if (rel > off) off = rel;
            if (rel < 1e-17) continue;
            double zeta = (beta - alpha) / (2.0 * gamma);
            double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
            double c = 1.0 / sqrt(1.0 + t * t);
            double s = c * t;
            for (int r = 0; r < 3; ++r) {
                double ap = a[r][p], aq = a[r][q];
                a[r][p] = c * ap - s * aq;
                a[r][q] = s * ap + c * aq;
                double vp = v[r][p], vq = v[r][q];
                v[r][p] = c * vp - s * vq;
                v[r][q] = s * vp + c * vq;
            }
        }
        if (off < 1e-15) break;
    }
    double sig[3];
    int order[3] = {0, 1, 2};
    for (int c = 0; c < 3; ++c) sig[c] = sqrt(a[0][c] * a[0][c] + a[1][c] * a[1][c] + a[2][c] * a[2][c]);
    for (int i = 0; i < 3; ++i)
        for (int j = i + 1; j < 3; ++j)
            if (sig[order[j]] > sig[order[i]]) { int t = order[i]; order[i] = order[j]; order[j] = t; }
    double U[3][3], VV[3][3], S[3];
    for (int k = 0; k < 3; ++k) {
        int c = order[k];
        S[k] = sig[c];
        for (int r = 0; r < 3; ++r) {
            VV[r][k] = v[r][c];
            U[r][k] = (sig[c] > 1e-300) ? a[r][c] / sig[c] : 0.0;
        }
    }
    /* Complete U for zero singular values (rank-deficient F). */
    double smax = S[0] > 0 ? S[0] : 1.0;
    if (S[1] <= 1e-300 * smax || S[1] == 0.0) {
        /* pick any unit vector orthogonal to U0 */
        double ux = U[0][0], uy = U[1][0], uz = U[2][0];
        double ox, oy, oz;
        if (fabs(ux) < 0.9) { ox = 0; oy = -uz; oz = uy; } else { ox = uz; oy = 0; oz = -ux; }
        double on = sqrt(ox * ox + oy * oy + oz * oz);
        if (on == 0) { ox = 1; oy = 0; oz = 0; on = 1; }
        U[0][1] = ox / on; U[1][1] = oy / on; U[2][1] = oz / on;
    }
    if (S[2] <= 1e-300 * smax || S[2] == 0.0) {
        U[0][2] = U[1][0] * U[2][1] - U[2][0] * U[1][1];
        U[1][2] = U[2][0] * U[0][1] - U[0][0] * U[2][1];
        U[2][2] = U[0][0] * U[1][1] - U[1][0] * U[0][1];
    }
    svd3 out;
    out.u = M(V((REAL)U[0][0], (REAL)U[1][0], (REAL)U[2][0]), V((REAL)U[0][1], (REAL)U[1][1], (REAL)U[2][1]),
              V((REAL)U[0][2], (REAL)U[1][2], (REAL)U[2][2]));
    out.s = V((REAL)S[0], (REAL)S[1], (REAL)S[2]);
    /* vt = V^T: column j of vt holds row j of V^T... i.e. vt[r][c] = V[c][r] */
    out.vt = M(V((REAL)VV[0][0], (REAL)VV[0][1], (REAL)VV[0][2]), V((REAL)VV[1][0], (REAL)VV[1][1], (REAL)VV[1][2]),
               V((REAL)VV[2][0], (REAL)VV[2][1], (REAL)VV[2][2]));
    return out;
}

/* ------------------------------------------------------------------------ */
/* Constitutive models: src_mpm_shaders/models/                              */
/* ------------------------------------------------------------------------ */

enum { MODEL_ELASTIC_LINEAR = 0, MODEL_ELASTIC_NEO_HOOKEAN = 1, MODEL_SAND_LINEAR = 2,
       MODEL_SAND_NEO_HOOKEAN = 3, MODEL_FLUID = 4, MODEL_SNOW = 5 };

/* linear_elasticity.rs:114-138 corotated Kirchhoff stress. */
static m3 linear_stress(REAL lambda, REAL mu, m3 F) {
    svd3 d = svd(F);
    REAL j = d.s.x * d.s.y * d.s.z;
    v3 ms = vsub(d.s, vsplat(1));
    m3 rec = mm(mm(d.u, mdiag(ms)), d.vt);
    REAL diag_val = lambda * (j - (REAL)1.0) * j;
    m3 res = mscale(mm(rec, mtr(F)), (REAL)2.0 * mu);
    res.c0.x += diag_val;
    res.c1.y += diag_val;
    res.c2.z += diag_val;
    return res;
}

/* neo_hookean_elasticity.rs:26-39 */
static m3 neo_hookean_stress(REAL lambda, REAL mu, m3 F) {
    REAL j = fmaxr(mdet(F), (REAL)1.0e-10);
    REAL diag_val = lambda * log(j) - mu;
    m3 st = mscale(mm(F, mtr(F)), mu);
    st.c0.x += diag_val;
    st.c1.y += diag_val;
    st.c2.z += diag_val;
    return st;
}

/* fluid.rs:54-85 */
static REAL fluid_pressure(const REAL *p, REAL j) {
    /* p = [bulk_modulus, gamma, viscosity, cfl_coeff, tensile_stiffness] */
    j = fmaxr(j, (REAL)1.0e-6);
    if (j <= (REAL)1.0) {
        REAL ratio = exp(-p[1] * log(j));
        return p[0] * (ratio - (REAL)1.0);
    }
    return -p[0] * p[4] * (j - (REAL)1.0);
}
static m3 fluid_stress(const REAL *p, m3 F, m3 strain_rate) {
    REAL j = fmaxr(mdet(F), (REAL)1.0e-6);
    /* models/utils.rs:241-283 deviatoric part */
    REAL sph = mtrace(strain_rate) / (REAL)3.0;
    m3 dev = strain_rate;
    dev.c0.x -= sph;
    dev.c1.y -= sph;
    dev.c2.z -= sph;
    m3 st = mscale(dev, (REAL)2.0 * p[2] * j);
    REAL diag_val = -fluid_pressure(p, j) * j;
    st.c0.x += diag_val;
    st.c1.y += diag_val;
    st.c2.z += diag_val;
    return st;
}

/* drucker_prager.rs:64-67 */
static REAL dp_alpha(const REAL *pl, REAL q) {
    /* pl = [ha, hb, hc, hd, lambda, mu, cohesion] */
    REAL angle = pl[0] + (pl[1] * q - pl[3]) * exp(-pl[2] * q);
    REAL s_angle = sin(angle);
    return sqrt((REAL)2.0 / (REAL)3.0) * ((REAL)2.0 * s_angle) / ((REAL)3.0 - s_angle);
}

/* drucker_prager.rs:121-167 (3D return mapping on log singular values). */
static int dp_project_sv(const REAL *pl, v3 s, REAL log_vol_gain, REAL alpha, v3 *sv_out, REAL *hard_out) {
    const REAL d = (REAL)3.0;
    v3 strain = vadd(V(log(s.x), log(s.y), log(s.z)), vsplat(log_vol_gain / d));
    REAL tr = strain.x + strain.y + strain.z;
    v3 dev = vsub(strain, vsplat(tr / d));
    REAL shifted = tr - pl[6];
    if (shifted > (REAL)0.0 || (dev.x == 0 && dev.y == 0 && dev.z == 0)) {
        *sv_out = vsplat(exp(pl[6] / d));
        *hard_out = vlen(strain);
        return 1;
    }
    REAL dnorm = vlen(dev);
    REAL gamma = dnorm + (d * pl[4] + (REAL)2.0 * pl[5]) / ((REAL)2.0 * pl[5]) * shifted * alpha;
    if (gamma <= (REAL)0.0) {
        *sv_out = vsplat(0);
        *hard_out = 0;
        return 0;
    }
    v3 h = vsub(strain, vmul(dev, gamma / dnorm));
    *sv_out = V(exp(h.x), exp(h.y), exp(h.z));
    *hard_out = gamma;
    return 1;
}

/* drucker_prager.rs:224-267 project(); state = [pdet, hardening, log_vol_gain]. */
static m3 dp_project(const REAL *pl, REAL *state, m3 F) {
    if (pl[4] == (REAL)0.0) return F;
    svd3 d = svd(F);
    REAL alpha = dp_alpha(pl, state[1]);
    v3 sv;
    REAL hard;
    int valid = dp_project_sv(pl, d.s, state[2], alpha, &sv, &hard);
    if (!valid) return F;
    REAL prev_det = d.s.x * d.s.y * d.s.z;
    REAL new_det = sv.x * sv.y * sv.z;
    REAL npdet = state[0] * prev_det / new_det;
    REAL nlvg = state[2] + log(prev_det) - log(new_det);
    REAL nhard = state[1] + hard;
    state[0] = npdet;
    state[1] = nhard;
    state[2] = nlvg;
    return mm(mm(d.u, mdiag(sv)), d.vt);
}

/* snow.rs:452-488; state = [plastic_det]; pl = [crit_compression, crit_stretch, hardening]. */
static m3 snow_project(const REAL *pl, REAL *state, m3 F, REAL *hardening) {
    if (pl[0] <= (REAL)0.0 && pl[1] <= (REAL)0.0) {
        *hardening = exp(pl[2] * ((REAL)1.0 - state[0]));
        return F;
    }
    svd3 d = svd(F);
    REAL lo = (REAL)1.0 - pl[0];
    REAL hi = (REAL)1.0 + pl[1];
    v3 cl = vclamp(d.s, lo, hi);
    REAL prev_det = d.s.x * d.s.y * d.s.z;
    REAL new_det = cl.x * cl.y * cl.z;
    REAL pdet = rclamp(state[0] * prev_det / new_det, (REAL)0.1, (REAL)4.0);
    state[0] = pdet;
    *hardening = exp(pl[2] * ((REAL)1.0 - pdet));
    return mm(mm(d.u, mdiag(cl)), d.vt);
}

/* models/default.rs:208-264 DefaultParticleModel::update. `w` holds the 24
 * model words as REAL (state words updated in place). Returns tau. */
static m3 model_update(uint32_t tag, REAL *w, m3 *F, m3 vel_grad) {
    switch (tag) {
    case MODEL_ELASTIC_LINEAR:
        return linear_stress(w[0], w[1], *F);
    case MODEL_ELASTIC_NEO_HOOKEAN:
        return neo_hookean_stress(w[0], w[1], *F);
    case MODEL_SAND_LINEAR: {
        /* layout default.rs:158-166: state[0..3] plastic[3..10] elastic[10..13] */
        *F = dp_project(&w[3], &w[0], *F);
        return linear_stress(w[10], w[11], *F);
    }
    case MODEL_SAND_NEO_HOOKEAN: {
        *F = dp_project(&w[3], &w[0], *F);
        return neo_hookean_stress(w[10], w[11], *F);
    }
    case MODEL_FLUID: {
        m3 sr = mscale(madd(vel_grad, mtr(vel_grad)), (REAL)0.5);
        return fluid_stress(&w[0], *F, sr);
    }
    case MODEL_SNOW: {
        /* layout default.rs:92-104: state[0] plastic[1..4] elastic[4..7] */
        REAL hard;
        *F = snow_project(&w[1], &w[0], *F, &hard);
        return linear_stress(w[4] * hard, w[5] * hard, *F);
    }
    default:
        return mzero();
    }
}

/* ------------------------------------------------------------------------ */
/* Colliders: shapes, projections, boundary conditions                      */
/* ------------------------------------------------------------------------ */

enum { SHAPE_BALL = 0, SHAPE_CUBOID = 1, SHAPE_CAPSULE = 2, SHAPE_TRIMESH = 6 };
enum { BC_STICK = 0, BC_SLIP = 1, BC_SEPARATE = 2, BC_NON_REFLECTING = 3 };

typedef struct {
    uint32_t type;
    REAL a[4], b[4], c[4];  /* Shape vec4s (shape.rs:29-73); a[3] holds the tag bits */
    pose3 pose;
    v3 linvel, angvel;      /* Velocity (dynamics/body.rs:216-225) */
    v3 local_com;           /* local centre of mass (for velocity_at_point) */
    v3 com;                 /* world centre of mass, refreshed each step */
    uint32_t bc_type;
    REAL bc_friction;
    /* trimesh: local-space triangles */
    uint32_t tri_first, tri_count;
} collider_t;

typedef struct { v3 point; int inside; } proj_t;

/* parry3d Ball::project_local_point, solid = false. */
static proj_t ball_project_local(REAL radius, v3 pt) {
    proj_t r;
    REAL d2 = vdot(pt, pt);
    r.inside = d2 <= radius * radius;
    r.point = vmul(pt, radius / sqrt(d2));
    return r;
}

/* parry3d Aabb::project_local_point (solid = false), cuboid = centred Aabb. */
static proj_t cuboid_project_local(v3 half, v3 pt) {
    v3 mins = vneg(half), maxs = half;
    v3 mins_pt = vsub(mins, pt);
    v3 pt_maxs = vsub(pt, maxs);
    v3 shift = vsub(V(fmaxr(mins_pt.x, 0), fmaxr(mins_pt.y, 0), fmaxr(mins_pt.z, 0)),
                    V(fmaxr(pt_maxs.x, 0), fmaxr(pt_maxs.y, 0), fmaxr(pt_maxs.z, 0)));
    proj_t r;
    int inside = (shift.x == 0 && shift.y == 0 && shift.z == 0);
    if (!inside) {
        r.inside = 0;
        r.point = vadd(pt, shift);
        return r;
    }
    REAL best = -MAX_FLT * (REAL)1e10;
    int is_mins = 0, best_id = 0;
    for (int i = 0; i < 3; ++i) {
        REAL mp = vget(mins_pt, i), pm = vget(pt_maxs, i);
        if (mp < pm) {
            if (pm > best) { best_id = i; is_mins = 0; best = pm; }
        } else if (mp > best) {
            best_id = i; is_mins = 1; best = mp;
        }
    }
    v3 s = V(0, 0, 0);
    REAL val = is_mins ? best : -best;
    if (best_id == 0) s.x = val; else if (best_id == 1) s.y = val; else s.z = val;
    r.inside = 1;
    r.point = vadd(pt, s);
    return r;
}

/* src_rbd_shaders/shapes/segment.rs project_local_point (closest point on a segment). */
static v3 segment_project_local(v3 a, v3 b, v3 pt) {
    v3 ab = vsub(b, a);
    v3 ap = vsub(pt, a);
    REAL ab_ap = vdot(ab, ap);
    REAL sqnab = vdot(ab, ab);
    if (ab_ap <= 0) return a;
    if (ab_ap >= sqnab) return b;
    REAL u = ab_ap / sqnab;
    return vadd(a, vmul(ab, u));
}

/* capsule.rs:62-81 project_local_point_on_boundary. */
static proj_t capsule_project_local(v3 a, v3 b, REAL radius, v3 pt) {
    v3 pa = segment_project_local(a, b, pt);
    v3 dproj = vsub(pt, pa);
    REAL d = vlen(dproj);
    proj_t r;
    if (d > 0) {
        r.inside = d <= radius;
        r.point = vadd(pa, vmul(dproj, radius / d));
    } else {
        v3 axis = vsub(b, a);
        REAL al = vlen(axis);
        v3 n = vdiv(axis, al);
        /* capsule.rs:164-173 any_orthogonal_vector: some unit vector orthogonal
         * to the axis (the exact basis choice only matters for points lying on
         * the axis itself). */
        v3 o = (fabs(n.x) > fabs(n.y)) ? V(-n.z, 0, n.x) : V(0, n.z, -n.y);
        o = vdiv(o, vlen(o));
        r.inside = 1;
        r.point = vadd(pa, vmul(o, radius));
    }
    return r;
}

/* solver/boundary_condition.rs:165-201 */
static v3 bc_project(uint32_t ty, REAL friction, v3 vel, v3 n) {
    if (ty == BC_STICK) return V(0, 0, 0);
    if (ty == BC_SLIP) {
        REAL nv = vdot(vel, n);
        return vsub(vel, vmul(n, nv));
    }
    if (ty == BC_SEPARATE) {
        REAL nv = vdot(vel, n);
        if (nv < 0) {
            v3 t = vsub(vel, vmul(n, nv));
            REAL tl = vlen(t);
            v3 tdir = tl > (REAL)1.0e-8 ? vdiv(t, tl) : V(0, 0, 0);
            REAL pl = tl + friction * nv;
            pl = pl > 0 ? pl : 0;
            return vmul(tdir, pl);
        }
        return vel;
    }
    return vel;
}

/* dynamics/body.rs:239-250 */
static inline v3 velocity_at_point(const collider_t *c, v3 p) {
    return vadd(c->linvel, vcross(c->angvel, vsub(p, c->com)));
}

/* ------------------------------------------------------------------------ */
/* Scene                                                                     */
/* ------------------------------------------------------------------------ */

typedef struct {
    /* particles (SoA) */
    uint32_t n;
    v3 *pos, *vel;
    m3 *aff, *F;
    REAL *vgd, *mass, *init_volume, *damping;
    uint32_t *enabled, *fixed, *tag;
    REAL *words; /* n * 24 */
    REAL *bfric; /* boundary_friction */
    float *init_radius, *phase; /* render-only properties (ParticleProperties) */
    uint32_t *group_id;
    /* particle Cdf (solver/particle.rs:35-50): normal, signed distance, rigid velocity, affinity bits */
    v3 *cdf_normal, *cdf_rigid_vel;
    REAL *cdf_sd;
    uint32_t *cdf_aff;
    /* params */
    v3 gravity;
    REAL dt;
    REAL dx;
    int use_cpic;
    /* grid */
    uint32_t capacity; /* blocks and hash slots (power of two) */
    uint32_t *hstate, *hvalue, *howner;
    header_t *hdr;
    uint32_t num_blocks;
    node_t *nodes;
    uint32_t *sorted;
    uint32_t *scan;
    /* colliders */
    uint32_t ncol;
    collider_t *col;
    v3 *tri; /* 3 vertices per triangle, local frame of the owning trimesh */
    uint32_t ntri;
    /* CPIC rigid particles: surface samples of the trimesh colliders
     * (solver/particle.rs:296-349), local and world positions, owning
     * collider and triangle (index into `tri`), the block-activation flag
     * and the block-sorted list with extras. */
    uint32_t nrp;
    int rp_dirty;
    v3 *rp_local, *rp_world;
    uint32_t *rp_col, *rp_tri;
    uint8_t *rp_need;
    uint32_t *rp_sorted;
    /* diagnostics */
    uint32_t status;
} scene_t;

enum { ORC_STATUS_HASH_FULL = 1u, ORC_STATUS_MISSING_BLOCK = 2u };

static void *xcalloc(size_t n, size_t s) { return calloc(n ? n : 1, s ? s : 1); }

scene_t *orc_create(uint32_t n, double dx, uint32_t grid_capacity) {
    scene_t *s = (scene_t *)xcalloc(1, sizeof(scene_t));
    s->n = n;
    s->dx = (REAL)dx;
    uint32_t cap = 1;
    while (cap < grid_capacity) cap <<= 1;
    s->capacity = cap;
    s->pos = xcalloc(n, sizeof(v3));
    s->vel = xcalloc(n, sizeof(v3));
    s->aff = xcalloc(n, sizeof(m3));
    s->F = xcalloc(n, sizeof(m3));
    s->vgd = xcalloc(n, sizeof(REAL));
    s->mass = xcalloc(n, sizeof(REAL));
    s->init_volume = xcalloc(n, sizeof(REAL));
    s->damping = xcalloc(n, sizeof(REAL));
    s->enabled = xcalloc(n, sizeof(uint32_t));
    s->bfric = xcalloc(n, sizeof(REAL));
    s->init_radius = xcalloc(n, sizeof(float));
    s->phase = xcalloc(n, sizeof(float));
    s->group_id = xcalloc(n, sizeof(uint32_t));
    for (uint32_t i = 0; i < n; ++i) s->bfric[i] = (REAL)1.0;
    s->cdf_normal = xcalloc(n, sizeof(v3));
    s->cdf_rigid_vel = xcalloc(n, sizeof(v3));
    s->cdf_sd = xcalloc(n, sizeof(REAL));
    s->cdf_aff = xcalloc(n, sizeof(uint32_t));
    s->fixed = xcalloc(n, sizeof(uint32_t));
    s->tag = xcalloc(n, sizeof(uint32_t));
    s->words = xcalloc((size_t)n * MODEL_WORDS, sizeof(REAL));
    s->hstate = xcalloc(cap, sizeof(uint32_t));
    s->hvalue = xcalloc(cap, sizeof(uint32_t));
    s->howner = xcalloc(cap, sizeof(uint32_t));
    s->hdr = xcalloc(cap, sizeof(header_t));
    s->nodes = xcalloc((size_t)cap * 64, sizeof(node_t));
    s->sorted = xcalloc((size_t)n * 8, sizeof(uint32_t));
    s->scan = xcalloc(cap, sizeof(uint32_t));
    for (uint32_t i = 0; i < cap; ++i) s->hstate[i] = NONE_U32;
    s->dt = (REAL)(1.0 / 60.0);
    return s;
}

void orc_destroy(scene_t *s) {
    if (!s) return;
    free(s->pos); free(s->vel); free(s->aff); free(s->F); free(s->vgd); free(s->mass);
    free(s->init_volume); free(s->damping); free(s->enabled); free(s->fixed); free(s->tag);
    free(s->bfric); free(s->init_radius); free(s->phase); free(s->group_id); free(s->cdf_normal); free(s->cdf_rigid_vel); free(s->cdf_sd); free(s->cdf_aff);
    free(s->words); free(s->hstate); free(s->hvalue); free(s->howner); free(s->hdr);
    free(s->nodes); free(s->sorted); free(s->scan); free(s->col); free(s->tri);
    free(s->rp_local); free(s->rp_world); free(s->rp_col); free(s->rp_tri); free(s->rp_need); free(s->rp_sorted);
    free(s);
}

static m3 load_m3(const float *p) {
    return M(V(p[0], p[1], p[2]), V(p[3], p[4], p[5]), V(p[6], p[7], p[8]));
}
static void store_m3(float *p, m3 m) {
    p[0] = (float)m.c0.x; p[1] = (float)m.c0.y; p[2] = (float)m.c0.z;
    p[3] = (float)m.c1.x; p[4] = (float)m.c1.y; p[5] = (float)m.c1.z;
    p[6] = (float)m.c2.x; p[7] = (float)m.c2.y; p[8] = (float)m.c2.z;
}

/* Loads particle state. Matrices are column-major 9 floats; `model` is
 * tag + 24 words per particle (GpuParticleModel, models/default.rs:41-44). */
void orc_set_particles(scene_t *s, const float *pos, const float *vel, const float *aff, const float *F,
                       const float *vgd, const float *mass, const float *init_volume, const float *damping,
                       const uint32_t *enabled, const uint32_t *fixed, const uint32_t *model) {
    for (uint32_t i = 0; i < s->n; ++i) {
        s->pos[i] = V(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
        s->vel[i] = V(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2]);
        s->aff[i] = load_m3(aff + 9 * (size_t)i);
        s->F[i] = load_m3(F + 9 * (size_t)i);
        s->vgd[i] = vgd[i];
        s->mass[i] = mass[i];
        s->init_volume[i] = init_volume[i];
        s->damping[i] = damping[i];
        s->enabled[i] = enabled[i];
        s->fixed[i] = fixed[i];
        s->tag[i] = model[25 * (size_t)i];
        for (int k = 0; k < MODEL_WORDS; ++k) s->words[(size_t)i * MODEL_WORDS + k] = bits2f(model[25 * (size_t)i + 1 + k]);
    }
}

void orc_set_boundary_friction(scene_t *s, const float *bf) {
    for (uint32_t i = 0; i < s->n; ++i) s->bfric[i] = bf[i];
}

void orc_set_render_props(scene_t *s, const float *init_radius, const float *phase, const uint32_t *group_id) {
    for (uint32_t i = 0; i < s->n; ++i) {
        s->init_radius[i] = init_radius[i];
        s->phase[i] = phase[i];
        s->group_id[i] = group_id[i];
    }
}

static float f2bitsf(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

/* Particle Cdf: normal xyz, signed distance, rigid velocity xyz, affinity bits (as float bits). */
void orc_get_cdf(const scene_t *s, float *out8) {
    for (uint32_t i = 0; i < s->n; ++i) {
        float *o = out8 + 8 * (size_t)i;
        o[0] = (float)s->cdf_normal[i].x; o[1] = (float)s->cdf_normal[i].y; o[2] = (float)s->cdf_normal[i].z;
        o[3] = (float)s->cdf_sd[i];
        o[4] = (float)s->cdf_rigid_vel[i].x; o[5] = (float)s->cdf_rigid_vel[i].y; o[6] = (float)s->cdf_rigid_vel[i].z;
        o[7] = f2bitsf(s->cdf_aff[i]);
    }
}

void orc_get_particles(const scene_t *s, float *pos, float *vel, float *aff, float *F, float *vgd, float *mass,
                       uint32_t *enabled, uint32_t *model) {
    for (uint32_t i = 0; i < s->n; ++i) {
        if (pos) { pos[3 * i] = (float)s->pos[i].x; pos[3 * i + 1] = (float)s->pos[i].y; pos[3 * i + 2] = (float)s->pos[i].z; }
        if (vel) { vel[3 * i] = (float)s->vel[i].x; vel[3 * i + 1] = (float)s->vel[i].y; vel[3 * i + 2] = (float)s->vel[i].z; }
        if (aff) store_m3(aff + 9 * (size_t)i, s->aff[i]);
        if (F) store_m3(F + 9 * (size_t)i, s->F[i]);
        if (vgd) vgd[i] = (float)s->vgd[i];
        if (mass) mass[i] = (float)s->mass[i];
        if (enabled) enabled[i] = s->enabled[i];
        if (model) {
            model[25 * (size_t)i] = s->tag[i];
            for (int k = 0; k < MODEL_WORDS; ++k)
                model[25 * (size_t)i + 1 + k] = f2bits((float)s->words[(size_t)i * MODEL_WORDS + k]);
        }
    }
}

/* Double-precision readback (positions) for the FP64 comparisons. */
void orc_get_positions_f64(const scene_t *s, double *pos) {
    for (uint32_t i = 0; i < s->n; ++i) {
        pos[3 * i] = (double)s->pos[i].x; pos[3 * i + 1] = (double)s->pos[i].y; pos[3 * i + 2] = (double)s->pos[i].z;
    }
}

void orc_set_params(scene_t *s, const float *gravity, float dt) {
    s->gravity = V(gravity[0], gravity[1], gravity[2]);
    s->dt = dt;
}

void orc_set_use_cpic(scene_t *s, int on) { s->use_cpic = on; s->rp_dirty = 1; }

/* Collider table.  Per collider, 32 floats:
 *   [0..4)  shape a, [4..8) shape b, [8..12) shape c      (Shape, shape.rs:29-73)
 *   [12..16) rotation quaternion x,y,z,w, [16..19) translation (Pose3)
 *   [19..22) linear velocity, [22..25) angular velocity   (Velocity)
 *   [25..28) local centre of mass
 *   [28] boundary condition type (u32 bits), [29] friction
 *   [30] first triangle (u32 bits), [31] triangle count (u32 bits)
 * The shape type is the bit pattern of a[3] (shape.rs:69-72). */
void orc_set_colliders(scene_t *s, uint32_t ncol, const float *desc, uint32_t ntri, const float *tri_vertices) {
    free(s->col);
    free(s->tri);
    s->ncol = ncol;
    s->col = xcalloc(ncol, sizeof(collider_t));
    s->ntri = ntri;
    s->tri = xcalloc((size_t)ntri * 3, sizeof(v3));
    for (uint32_t i = 0; i < ncol; ++i) {
        const float *d = desc + 32 * (size_t)i;
        collider_t *c = &s->col[i];
        for (int k = 0; k < 4; ++k) { c->a[k] = d[k]; c->b[k] = d[4 + k]; c->c[k] = d[8 + k]; }
        c->type = f2bits(d[3]);
        c->pose.rot.x = d[12]; c->pose.rot.y = d[13]; c->pose.rot.z = d[14]; c->pose.rot.w = d[15];
        c->pose.tra = V(d[16], d[17], d[18]);
        c->linvel = V(d[19], d[20], d[21]);
        c->angvel = V(d[22], d[23], d[24]);
        c->local_com = V(d[25], d[26], d[27]);
        c->bc_type = f2bits(d[28]);
        c->bc_friction = d[29];
        c->tri_first = f2bits(d[30]);
        c->tri_count = f2bits(d[31]);
        c->com = pose_apply(c->pose, c->local_com);
    }
    for (uint32_t t = 0; t < ntri * 3; ++t)
        s->tri[t] = V(tri_vertices[3 * t], tri_vertices[3 * t + 1], tri_vertices[3 * t + 2]);
    s->rp_dirty = 1;
}

void orc_set_collider_velocity(scene_t *s, uint32_t i, const float *lin, const float *ang) {
    if (i >= s->ncol) return;
    s->col[i].linvel = V(lin[0], lin[1], lin[2]);
    s->col[i].angvel = V(ang[0], ang[1], ang[2]);
}

void orc_get_collider_pose(const scene_t *s, uint32_t i, float *out7) {
    if (i >= s->ncol) return;
    const collider_t *c = &s->col[i];
    out7[0] = (float)c->pose.rot.x; out7[1] = (float)c->pose.rot.y; out7[2] = (float)c->pose.rot.z;
    out7[3] = (float)c->pose.rot.w; out7[4] = (float)c->pose.tra.x; out7[5] = (float)c->pose.tra.y;
    out7[6] = (float)c->pose.tra.z;
}

/* ------------------------------------------------------------------------ */
/* Rigid particles of trimesh colliders (CPIC):                              */
/* src_mpm/sampling/sample_trimesh.rs, in f32 as the reference samples       */
/* ------------------------------------------------------------------------ */

#define SAMPLE_EPS 1.0e-5f  /* sample_trimesh.rs:12 */

typedef struct { float x, y, z; } f3;
static inline f3 F3(float x, float y, float z) { f3 r = {x, y, z}; return r; }
static inline f3 fsub(f3 a, f3 b) { return F3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline f3 fadd(f3 a, f3 b) { return F3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline f3 fmulv(f3 a, float s) { return F3(a.x * s, a.y * s, a.z * s); }
static inline f3 fdivv(f3 a, float s) { return F3(a.x / s, a.y / s, a.z / s); }
static inline float fdot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float flen3(f3 a) { return sqrtf(fdot3(a, a)); }
/* Rust `f32 as u32` / `as usize` for the step counts: saturating, NaN -> 0. */
static inline uint32_t f_to_count(float f) { return !(f > 0.0f) ? 0u : (f >= 4294967295.0f ? 0xFFFFFFFFu : (uint32_t)f); }

typedef struct { f3 *pt; uint32_t *tri; uint32_t len, cap; } samples_t;
static void samples_push(samples_t *b, f3 p, uint32_t tri) {
    if (b->len == b->cap) {
        b->cap = b->cap ? 2 * b->cap : 1024;
        b->pt = realloc(b->pt, sizeof(f3) * b->cap);
        b->tri = realloc(b->tri, sizeof(uint32_t) * b->cap);
    }
    b->pt[b->len] = p;
    b->tri[b->len++] = tri;
}

/* sample_trimesh.rs:116-138 sample_edge: points every xy_spacing/sqrt(2)
 * from a (excluded) toward b. */
static void sample_edge(f3 a, f3 b, float xy_spacing, uint32_t tri, samples_t *out) {
    f3 ab = fsub(b, a);
    float len = flen3(ab);
    if (len > SAMPLE_EPS) {
        f3 dir = fdivv(ab, len);
        float spacing = xy_spacing / sqrtf(2.0f);
        uint32_t nsteps = f_to_count(ceilf(len / spacing));
        for (uint32_t i = 1; i < nsteps; ++i) samples_push(out, fadd(a, fmulv(dir, spacing * (float)i)), tri);
    }
}

/* sample_trimesh.rs:140-231 sample_triangle: the longest edge is the base;
 * rows perpendicular to it every spacing, points along each row every
 * spacing, none on the base, the row ends or the vertices. */
static void sample_triangle(f3 a, f3 b, f3 c, float xy_spacing, uint32_t tri, samples_t *out) {
    float d_ab = flen3(fsub(b, a)), d_bc = flen3(fsub(c, b)), d_ca = flen3(fsub(a, c));
    float mx = fmaxf(fmaxf(d_ab, d_bc), d_ca);
    if (mx == d_bc) { f3 t = a; a = b; b = c; c = t; }
    else if (mx == d_ca) { f3 t = a; a = c; c = b; b = t; }
    f3 ac = fsub(c, a), base = fsub(b, a);
    float base_length = flen3(base);
    f3 base_dir = fdivv(base, base_length);
    float spacing = xy_spacing / sqrtf(2.0f);
    float base_steps = ceilf(base_length / spacing);
    f3 base_step = fmulv(base_dir, spacing);
    float ac_off = fdot3(ac, base_dir);
    float bc_off = base_length - ac_off;
    if (ac_off < SAMPLE_EPS || bc_off < SAMPLE_EPS || base_length < SAMPLE_EPS) return;
    f3 height = fsub(ac, fmulv(base_dir, ac_off));
    float height_length = flen3(height);
    f3 height_dir = fdivv(height, height_length);
    float tan_a = height_length / ac_off, tan_b = height_length / bc_off;
    uint32_t nb = f_to_count(base_steps);
    for (uint32_t i = 1; i < nb; ++i) {
        f3 bp = fadd(a, fmulv(base_step, (float)i));
        float h_ac = tan_a * flen3(fsub(a, bp));
        float h_bc = tan_b * flen3(fsub(b, bp));
        float hl = fminf(h_ac, h_bc);
        uint32_t nh = f_to_count(ceilf(hl / spacing));
        f3 hstep = fmulv(height_dir, spacing);
        for (uint32_t j = 1; j < nh; ++j) {
            f3 pp = fadd(bp, fmulv(hstep, (float)j));
            if (!isfinite(pp.x) || !isfinite(pp.y) || !isfinite(pp.z)) continue;
            samples_push(out, pp, tri);
        }
    }
}

/* Vertex identity of a triangle soup: equal position bits = one vertex (the
 * reference's meshes are indexed; a soup carries the index as the position). */
typedef struct { uint32_t *key; uint32_t *id; uint32_t mask, count; } vtab_t;
static uint32_t mix3(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t h = hash_key(a) ^ 0x9E3779B9u;
    h = hash_key(h ^ b) + 0x7F4A7C15u;
    return hash_key(h ^ c);
}
static uint32_t vtab_id(vtab_t *t, f3 p) {
    uint32_t k0, k1, k2;
    memcpy(&k0, &p.x, 4); memcpy(&k1, &p.y, 4); memcpy(&k2, &p.z, 4);
    uint32_t slot = mix3(k0, k1, k2) & t->mask;
    for (;;) {
        uint32_t *k = t->key + 3 * (size_t)slot;
        if (t->id[slot] == NONE_U32) {
            k[0] = k0; k[1] = k1; k[2] = k2;
            t->id[slot] = t->count++;
            return t->id[slot];
        }
        if (k[0] == k0 && k[1] == k1 && k[2] == k2) return t->id[slot];
        slot = (slot + 1) & t->mask;
    }
}
typedef struct { uint64_t *key; uint32_t mask; } etab_t;
/* sample_trimesh.rs:73-81: true the first time an (unordered) edge is seen. */
static int etab_insert(etab_t *t, uint32_t a, uint32_t b) {
    if (b > a) { uint32_t x = a; a = b; b = x; }
    uint64_t key = ((uint64_t)a << 32) | b;
    uint32_t slot = mix3(a, b, 0x51u) & t->mask;
    for (;;) {
        if (t->key[slot] == UINT64_MAX) { t->key[slot] = key; return 1; }
        if (t->key[slot] == key) return 0;
        slot = (slot + 1) & t->mask;
    }
}

/* sample_trimesh.rs:66-114 sample_mesh for every trimesh collider in
 * collider order (solver/particle.rs:305-346), sampling step = cell width. */
static void build_rigid_particles(scene_t *s) {
    free(s->rp_local); free(s->rp_world); free(s->rp_col); free(s->rp_tri); free(s->rp_need); free(s->rp_sorted);
    s->rp_local = s->rp_world = NULL;
    s->rp_col = s->rp_tri = s->rp_sorted = NULL;
    s->rp_need = NULL;
    s->nrp = 0;
    s->rp_dirty = 0;
    if (!s->use_cpic) return;
    samples_t all = {0};
    uint32_t *cols = NULL;
    size_t cols_cap = 0;
    const float step = (float)s->dx;
    for (uint32_t ci = 0; ci < s->ncol; ++ci) {
        const collider_t *c = &s->col[ci];
        if (c->type != SHAPE_TRIMESH) continue;
        uint32_t cap = 16;
        while (cap < 6 * c->tri_count + 16) cap <<= 1;
        vtab_t vt = {malloc(sizeof(uint32_t) * 3 * (size_t)cap), malloc(sizeof(uint32_t) * cap), cap - 1, 0};
        etab_t et = {malloc(sizeof(uint64_t) * cap), cap - 1};
        for (uint32_t i = 0; i < cap; ++i) { vt.id[i] = NONE_U32; et.key[i] = UINT64_MAX; }
        const uint32_t before = all.len;
        for (uint32_t t = c->tri_first; t < c->tri_first + c->tri_count; ++t) {
            f3 q[3];
            uint32_t vid[3];
            for (int k = 0; k < 3; ++k) {
                v3 v = s->tri[3 * (size_t)t + k];
                q[k] = F3((float)v.x, (float)v.y, (float)v.z);
                vid[k] = vtab_id(&vt, q[k]);
            }
            sample_triangle(q[0], q[1], q[2], step, t, &all);
            if (etab_insert(&et, vid[0], vid[1])) sample_edge(q[0], q[1], step, t, &all);
            if (etab_insert(&et, vid[1], vid[2])) sample_edge(q[1], q[2], step, t, &all);
            if (etab_insert(&et, vid[2], vid[0])) sample_edge(q[2], q[0], step, t, &all);
        }
        free(vt.key); free(vt.id); free(et.key);
        if (all.len > cols_cap) {
            cols_cap = all.cap;
            cols = realloc(cols, sizeof(uint32_t) * cols_cap);
        }
        for (uint32_t i = before; i < all.len; ++i) cols[i] = ci;
    }
    s->nrp = all.len;
    s->rp_local = xcalloc(s->nrp, sizeof(v3));
    s->rp_world = xcalloc(s->nrp, sizeof(v3));
    s->rp_col = xcalloc(s->nrp, sizeof(uint32_t));
    s->rp_tri = xcalloc(s->nrp, sizeof(uint32_t));
    s->rp_need = xcalloc(s->nrp, 1);
    s->rp_sorted = xcalloc((size_t)s->nrp * 8, sizeof(uint32_t));
    for (uint32_t i = 0; i < s->nrp; ++i) {
        s->rp_local[i] = V(all.pt[i].x, all.pt[i].y, all.pt[i].z);
        s->rp_world[i] = s->rp_local[i];  /* solver/particle.rs:272-276: world = local until the first step */
        s->rp_col[i] = cols[i];
        s->rp_tri[i] = all.tri[i];
    }
    free(all.pt); free(all.tri); free(cols);
}

uint32_t orc_num_rigid(scene_t *s) {
    if (s->rp_dirty) build_rigid_particles(s);
    return s->nrp;
}
/* Per rigid particle 5 floats: local position, collider (u32 bits), triangle
 * index inside its collider's range (u32 bits). */
void orc_get_rigid(scene_t *s, float *out5) {
    if (s->rp_dirty) build_rigid_particles(s);
    for (uint32_t i = 0; i < s->nrp; ++i) {
        float *o = out5 + 5 * (size_t)i;
        o[0] = (float)s->rp_local[i].x; o[1] = (float)s->rp_local[i].y; o[2] = (float)s->rp_local[i].z;
        o[3] = f2bitsf(s->rp_col[i]);
        o[4] = f2bitsf(s->rp_tri[i] - s->col[s->rp_col[i]].tri_first);
    }
}

/* rigid_particle_update.rs:9-31 gpu_transform_sample_points. */
static void transform_rigid_particles(scene_t *s) {
    for (uint32_t i = 0; i < s->nrp; ++i) s->rp_world[i] = pose_apply(s->col[s->rp_col[i]].pose, s->rp_local[i]);
}

/* ------------------------------------------------------------------------ */
/* Hash map ops, sequential (grid.rs:447-578)                                */
/* ------------------------------------------------------------------------ */

static uint32_t insertion_index(scene_t *s, i3 key) {
    uint32_t pk = pack_key(key);
    uint32_t mask = s->capacity - 1;
    uint32_t slot = hash_key(pk) & mask;
    for (uint32_t it = 0; it < s->capacity; ++it) {
        uint32_t old = s->hstate[slot];
        if (old == pk) return NONE_U32;
        if (old != NONE_U32) { slot = (slot + 1) & mask; continue; }
        s->hstate[slot] = pk;
        if (s->howner[slot] == 0) { s->howner[slot] = 1; return slot; }
        return NONE_U32;
    }
    s->status |= ORC_STATUS_HASH_FULL;
    return NONE_U32;
}

static uint32_t find_header(const scene_t *s, i3 key) {
    uint32_t pk = pack_key(key);
    uint32_t mask = s->capacity - 1;
    uint32_t slot = hash_key(pk) & mask;
    for (uint32_t it = 0; it < s->capacity; ++it) {
        uint32_t st = s->hstate[slot];
        if (st == pk) return s->hvalue[slot];
        if (st == NONE_U32) break;
        slot = (slot + 1) & mask;
    }
    return NONE_U32;
}

static void mark_active(scene_t *s, i3 key) {
    uint32_t slot = insertion_index(s, key);
    if (slot != NONE_U32) {
        uint32_t id = s->num_blocks++;
        header_t *h = &s->hdr[id];
        memset(h, 0, sizeof(*h));
        h->vid = key;
        s->hvalue[slot] = id;
    }
}

/* ------------------------------------------------------------------------ */
/* Sort: src_mpm/grid/grid.rs:26-191 + src_mpm_shaders/grid/sort.rs          */
/* ------------------------------------------------------------------------ */

/* sort.rs:56-62 extra bucket. */
static inline uint32_t extra_bucket(const uint32_t assoc[3], i3 bshift) {
    int32_t local = (int32_t)assoc[2] - bshift.z * 4;
    if (local < -2) local = -2;
    return NUM_PRIMARY_BUCKETS + (uint32_t)(local + 2);
}
static inline int spills(const uint32_t assoc[3], i3 bshift) {
    return (bshift.x == 0 || assoc[0] >= 2) && (bshift.y == 0 || assoc[1] >= 2) && (bshift.z == 0 || assoc[2] >= 2);
}

/* sort.rs:493-667: rigid particles per block (their own block, plus each
 * +1 neighbour their 3-cell range reaches when it exists; a particle whose
 * own block is missing is skipped), exclusive scan, placement in ascending
 * particle order. */
static void rigid_sort(scene_t *s) {
    const REAL dx = s->dx;
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) {
            uint32_t run = 0;
            for (uint32_t b = 0; b < s->num_blocks; ++b) {
                s->hdr[b].first_rigid = run;
                run += s->hdr[b].num_rigid;
                s->hdr[b].num_rigid = 0;
            }
        } else {
            for (uint32_t b = 0; b < s->num_blocks; ++b) s->hdr[b].num_rigid = 0;
        }
        for (uint32_t p = 0; p < s->nrp; ++p) {
            uint32_t h0 = find_header(s, block_of_point(dx, s->rp_world[p]));
            if (h0 == NONE_U32) continue;
            uint32_t assoc[3];
            assoc_in_block(dx, s->rp_world[p], assoc);
            uint32_t hs[8], nh = 0;
            hs[nh++] = h0;
            for (int i = 1; i < 8; ++i)
                if (spills(assoc, ASSOC_SHIFT[i]) && s->hdr[h0].nbh[i - 1] != NONE_U32) hs[nh++] = s->hdr[h0].nbh[i - 1];
            for (uint32_t k = 0; k < nh; ++k) {
                header_t *h = &s->hdr[hs[k]];
                if (pass == 1) s->rp_sorted[h->first_rigid + h->num_rigid] = p;
                h->num_rigid += 1;
            }
        }
    }
}

int orc_sort(scene_t *s) {
    const REAL dx = s->dx;
    /* grid.rs:660-685 reset_hmap */
    for (uint32_t i = 0; i < s->capacity; ++i) { s->hstate[i] = NONE_U32; s->howner[i] = 0; s->hvalue[i] = 0; }
    s->num_blocks = 0;
    /* sort.rs:104-121 touch primary blocks */
    for (uint32_t p = 0; p < s->n; ++p) mark_active(s, block_of_point(dx, s->pos[p]));
    /* grid.rs:694-700 capture; sort.rs:133-163 touch neighbour blocks */
    uint32_t nbase = s->num_blocks;
    for (uint32_t b = 0; b < nbase; ++b) {
        i3 vid = s->hdr[b].vid;
        for (int i = 1; i < 8; ++i) mark_active(s, i3add(vid, ASSOC_SHIFT[i]));
    }
    /* grid.rs:95-121: CPIC rigid particles whose own block is missing while
     * one of its +1 neighbours exists get their own block (sort.rs:200-249
     * marks them all first, sort.rs:165-198 then inserts). */
    if (s->use_cpic && s->nrp) {
        for (uint32_t p = 0; p < s->nrp; ++p) {
            i3 b0 = block_of_point(dx, s->rp_world[p]);
            int i = 0;
            for (; i < 8; ++i)
                if (find_header(s, i3add(b0, ASSOC_SHIFT[i])) != NONE_U32) break;
            s->rp_need[p] = (uint8_t)(i > 0 && i < 8);
        }
        for (uint32_t p = 0; p < s->nrp; ++p)
            if (s->rp_need[p]) mark_active(s, block_of_point(dx, s->rp_world[p]));
    }
    /* sort.rs:261-279 update_nbh_block_ids */
    for (uint32_t b = 0; b < s->num_blocks; ++b)
        for (int i = 0; i < NUM_NBH; ++i) s->hdr[b].nbh[i] = find_header(s, i3add(s->hdr[b].vid, ASSOC_SHIFT[i + 1]));
    /* sort.rs:287-349 update_block_particle_count */
    for (uint32_t p = 0; p < s->n; ++p) {
        i3 b0 = block_of_point(dx, s->pos[p]);
        uint32_t assoc[3];
        assoc_in_block(dx, s->pos[p], assoc);
        uint32_t h0 = find_header(s, b0);
        if (h0 == NONE_U32) { s->status |= ORC_STATUS_MISSING_BLOCK; continue; }
        s->hdr[h0].cursors[assoc[2]] += 1;
        for (int i = 1; i < 8; ++i) {
            i3 bs = ASSOC_SHIFT[i];
            if (spills(assoc, bs)) {
                uint32_t hi = s->hdr[h0].nbh[i - 1];
                if (hi == NONE_U32) { s->status |= ORC_STATUS_MISSING_BLOCK; continue; }
                s->hdr[hi].cursors[extra_bucket(assoc, bs)] += 1;
            }
        }
    }
    /* sort.rs:357-374 copy_particles_len_to_scan_value */
    for (uint32_t b = 0; b < s->num_blocks; ++b) {
        uint32_t t = 0;
        for (int k = 0; k < NUM_BUCKETS; ++k) t += s->hdr[b].cursors[k];
        s->scan[b] = t;
    }
    /* src_rbd/utils/prefix_sum.rs:112-136 exclusive scan with a leading 0
     * (over the active prefix; entries past it are never read). */
    {
        uint32_t run = 0;
        for (uint32_t b = 0; b < s->num_blocks; ++b) { uint32_t t = s->scan[b]; s->scan[b] = run; run += t; }
    }
    /* sort.rs:382-420 copy_scan_values_to_first_particles */
    for (uint32_t b = 0; b < s->num_blocks; ++b) {
        header_t *h = &s->hdr[b];
        uint32_t first = s->scan[b];
        h->first_particle = first;
        uint32_t running = first;
        for (int k = 0; k < NUM_BUCKETS; ++k) {
            if (k == NUM_PRIMARY_BUCKETS) h->num_particles = running - first;
            uint32_t c = h->cursors[k];
            h->cursors[k] = running;
            running += c;
        }
        h->num_particles_with_extras = running - first;
    }
    /* sort.rs:430-491 finalize_particles_sort */
    for (uint32_t p = 0; p < s->n; ++p) {
        i3 b0 = block_of_point(dx, s->pos[p]);
        uint32_t assoc[3];
        assoc_in_block(dx, s->pos[p], assoc);
        uint32_t h0 = find_header(s, b0);
        if (h0 == NONE_U32) continue;
        s->sorted[s->hdr[h0].cursors[assoc[2]]++] = p;
        for (int i = 1; i < 8; ++i) {
            i3 bs = ASSOC_SHIFT[i];
            if (spills(assoc, bs)) {
                uint32_t hi = s->hdr[h0].nbh[i - 1];
                if (hi == NONE_U32) continue;
                s->sorted[s->hdr[hi].cursors[extra_bucket(assoc, bs)]++] = p;
            }
        }
    }
    if (s->use_cpic && s->nrp) rigid_sort(s);
    return (int)s->status;
}

/* ------------------------------------------------------------------------ */
/* CPIC affinity bits (grid/grid.rs:593-645)                                 */
/* ------------------------------------------------------------------------ */

#define AFF_MASK 0x0000FFFFu
#define AFF_SIGN_SHIFT 16
static inline int aff_compatible(uint32_t a, uint32_t b) {
    uint32_t common = a & b & AFF_MASK;
    return ((a >> AFF_SIGN_SHIFT) & common) == ((b >> AFF_SIGN_SHIFT) & common);
}

/* ------------------------------------------------------------------------ */
/* P2G (gather form): solver/p2g.rs:64-351 (USE_CPIC: compatible and         */
/* incompatible sums, two-way impulses off as TWO_WAYS_COUPLING_ENABLED)     */
/* ------------------------------------------------------------------------ */

void orc_p2g(scene_t *s) {
    const REAL dx = s->dx;
    const REAL inv_dx = (REAL)1.0 / dx;
    const int64_t nb = (int64_t)s->num_blocks;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t bi = 0; bi < nb; ++bi) {
        const header_t *h = &s->hdr[bi];
        const i3 vid = h->vid;
        const uint32_t first = h->first_particle;
        const uint32_t num = h->num_particles_with_extras;
        const uint32_t last = first + num;
        const uint32_t primaries_end = first + h->num_particles;
        const uint32_t nchunks = (num + 63) / 64;
        /* one accumulator set per node of the block; tid = x + 4y + 16z */
        v3 acc_mv[64];
        REAL acc_m[64];
        for (int t = 0; t < 64; ++t) { acc_mv[t] = V(0, 0, 0); acc_m[t] = 0; }
        v3 acc_mvi[64];
        REAL acc_mi[64];
        for (int t = 0; t < 64; ++t) { acc_mvi[t] = V(0, 0, 0); acc_mi[t] = 0; }
        v3 spos[64], smom[64];
        REAL smass[64];
        m3 saff[64];
        int32_t szkey[64];
        uint32_t safn[64];
        for (uint32_t chunk = 0; chunk < nchunks; ++chunk) {
            uint32_t base = first + chunk * 64;
            uint32_t clen = (last - base) < 64 ? (last - base) : 64;
            for (uint32_t k = 0; k < clen; ++k) {
                uint32_t pid = s->sorted[base + k];
                v3 pt = s->pos[pid];
                safn[k] = s->cdf_aff[pid];
                v3 ac = assoc_cell_of(dx, pt);
                int32_t zk = r_to_i32(ac.z) - vid.z * 4;
                szkey[k] = zk < -2 ? -2 : zk;
                if (s->enabled[pid] != 0) {
                    spos[k] = pt;
                    smom[k] = vmul(s->vel[pid], s->mass[pid]);
                    smass[k] = s->mass[pid];
                    saff[k] = s->aff[pid];
                } else {
                    spos[k] = V(0, 0, 0);
                    smom[k] = V(0, 0, 0);
                    smass[k] = 0;
                    saff[k] = mzero();
                }
            }
            int32_t zmin = szkey[0], zmax = szkey[clen - 1];
            if (primaries_end > base && primaries_end < base + clen) {
                uint32_t b = primaries_end - base;
                if (szkey[b] < zmin) zmin = szkey[b];
                if (szkey[b - 1] > zmax) zmax = szkey[b - 1];
            }
            for (int tz = 0; tz < 4; ++tz) {
                if (!(tz >= zmin && tz <= zmax + 2)) continue;
                for (int ty = 0; ty < 4; ++ty)
                    for (int tx = 0; tx < 4; ++tx) {
                        int t = tx + 4 * ty + 16 * tz;
                        v3 cell_pos = vmul(V((REAL)(vid.x * 4 + tx), (REAL)(vid.y * 4 + ty), (REAL)(vid.z * 4 + tz)), dx);
                        const uint32_t node_aff = s->nodes[(size_t)bi * 64 + t].cdf_aff;
                        for (uint32_t p = 0; p < clen; ++p) {
                            v3 dpt = vsub(cell_pos, spos[p]);
                            REAL w = kernel_eval(dpt.x * inv_dx) * kernel_eval(dpt.y * inv_dx) * kernel_eval(dpt.z * inv_dx);
                            if (w != 0) {
                                v3 vc = vmul(vadd(mv(saff[p], dpt), smom[p]), w);
                                REAL mc = smass[p] * w;
                                /* p2g.rs:268-305: an incompatible particle feeds the node's second field */
                                if (s->use_cpic && !aff_compatible(safn[p], node_aff)) {
                                    acc_mvi[t] = vadd(acc_mvi[t], vc);
                                    acc_mi[t] += mc;
                                } else {
                                    acc_mv[t] = vadd(acc_mv[t], vc);
                                    acc_m[t] += mc;
                                }
                            }
                        }
                    }
            }
        }
        for (int t = 0; t < 64; ++t) {
            node_t *nd = &s->nodes[(size_t)bi * 64 + t];
            nd->mv = acc_mv[t];
            nd->mass = acc_m[t];
            nd->mv_incompat = acc_mvi[t];
            nd->mass_incompat = acc_mi[t];
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Grid update: solver/grid_update.rs:21-88 and grid_update_collide.rs       */
/* ------------------------------------------------------------------------ */

static inline v3 update_single_cell(const scene_t *s, v3 momentum, REAL mass) {
    REAL inv_mass = mass > 0 ? (REAL)1.0 / mass : (REAL)0.0;
    v3 v = vmul(vadd(momentum, vmul(s->gravity, mass * s->dt)), inv_mass);
    REAL lim = s->dx / s->dt;
    return vclamp(v, -lim, lim);
}

typedef struct { v3 normal; REAL distance; uint32_t closest; } collision_t;

static proj_t trimesh_project(const scene_t *s, const collider_t *c, v3 local_pt, REAL max_dist, int *valid);

/* grid_update_collide.rs:30-99 collide() */
static collision_t collide(const scene_t *s, v3 point) {
    REAL cap = s->dx * (REAL)1.5;
    collision_t col;
    col.normal = V(0, 0, 0);
    col.distance = MAX_FLT;
    col.closest = 0;
    for (uint32_t i = 0; i < s->ncol; ++i) {
        const collider_t *c = &s->col[i];
        proj_t pr;
        int valid = 1;
        if (c->type == SHAPE_TRIMESH) {
            /* pose.inverse() * point */
            quat ci = qconj(c->pose.rot);
            v3 itra = vneg(qrot(ci, c->pose.tra));
            v3 local = vadd(qrot(ci, point), itra);
            pr = trimesh_project(s, c, local, cap, &valid);
            pr.point = pose_apply(c->pose, pr.point);
        } else {
            v3 local = pose_inv_apply(c->pose, point);
            if (c->type == SHAPE_BALL) pr = ball_project_local(c->a[0], local);
            else if (c->type == SHAPE_CUBOID) pr = cuboid_project_local(V(c->a[0], c->a[1], c->a[2]), local);
            else if (c->type == SHAPE_CAPSULE)
                pr = capsule_project_local(V(c->a[0], c->a[1], c->a[2]), V(c->b[0], c->b[1], c->b[2]), c->b[3], local);
            else { pr.point = local; pr.inside = 0; }
            pr.point = pose_apply(c->pose, pr.point);
        }
        if (valid) {
            v3 dpt = vsub(pr.point, point);
            v3 ad = vabs(dpt);
            int within = ad.x <= cap && ad.y <= cap && ad.z <= cap;
            if (pr.inside || within) {
                REAL sign = pr.inside ? (REAL)-1.0 : (REAL)1.0;
                REAL distance = vlen(dpt);
                v3 normal = vdiv(dpt, distance * -sign);
                REAL sd = sign * distance;
                if (sd < col.distance) {
                    col.distance = sd;
                    col.normal = normal;
                    col.closest = i;
                }
            }
        }
    }
    return col;
}

void orc_grid_update(scene_t *s) {
    const int64_t nb = (int64_t)s->num_blocks;
#pragma omp parallel for schedule(static)
    for (int64_t bi = 0; bi < nb; ++bi) {
        const i3 vid = s->hdr[bi].vid;
        for (int t = 0; t < 64; ++t) {
            int tx = t & 3, ty = (t >> 2) & 3, tz = t >> 4;
            node_t *nd = &s->nodes[(size_t)bi * 64 + t];
            nd->mv = update_single_cell(s, nd->mv, nd->mass);
            nd->mv_incompat = update_single_cell(s, nd->mv_incompat, nd->mass_incompat);
            if (!s->use_cpic && s->ncol > 0) {
                v3 cell_pt = vmul(V((REAL)(vid.x * 4 + tx), (REAL)(vid.y * 4 + ty), (REAL)(vid.z * 4 + tz)), s->dx);
                collision_t col = collide(s, cell_pt);
                if (col.distance != MAX_FLT) {
                    const collider_t *c = &s->col[col.closest];
                    v3 bv = velocity_at_point(c, cell_pt);
                    v3 delta = vsub(nd->mv, bv);
                    REAL nv = vdot(delta, col.normal);
                    REAL margin = s->dx;
                    if (col.distance <= margin) {
                        nd->mv = vadd(bv, bc_project(c->bc_type, c->bc_friction, delta, col.normal));
                    } else if (-nv * s->dt > col.distance - margin) {
                        v3 excess = vmul(col.normal, nv + (col.distance - margin) / s->dt);
                        nd->mv = vsub(nd->mv, excess);
                    }
                }
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* G2P: solver/g2p.rs:42-347 with USE_CPIC = false                           */
/* ------------------------------------------------------------------------ */

/* Node velocity seen by block `vid` at shared-tile coordinate s in [0,6)^3. */
static inline v3 halo_vel(const scene_t *s, const uint32_t octant_hdr[8], int sx, int sy, int sz) {
    int ox = sx >= 4, oy = sy >= 4, oz = sz >= 4;
    uint32_t h = octant_hdr[ox * 4 + oy * 2 + oz];
    if (h == NONE_U32) return V(0, 0, 0);
    int lx = sx - 4 * ox, ly = sy - 4 * oy, lz = sz - 4 * oz;
    return s->nodes[(size_t)h * 64 + lx + 4 * ly + 16 * lz].mv;
}

static inline const node_t *halo_node(const scene_t *s, const uint32_t octant_hdr[8], int sx, int sy, int sz) {
    int ox = sx >= 4, oy = sy >= 4, oz = sz >= 4;
    uint32_t h = octant_hdr[ox * 4 + oy * 2 + oz];
    if (h == NONE_U32) return NULL;
    int lx = sx - 4 * ox, ly = sy - 4 * oy, lz = sz - 4 * oz;
    return &s->nodes[(size_t)h * 64 + lx + 4 * ly + 16 * lz];
}

void orc_g2p(scene_t *s) {
    const REAL dx = s->dx;
    const REAL inv_d = (REAL)4.0 / (dx * dx);
    const int64_t nb = (int64_t)s->num_blocks;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t bi = 0; bi < nb; ++bi) {
        const header_t *h = &s->hdr[bi];
        uint32_t oct[8];
        for (int o = 0; o < 8; ++o) oct[o] = find_header(s, i3add(h->vid, ASSOC_SHIFT[o]));
        for (uint32_t k = h->first_particle; k < h->first_particle + h->num_particles; ++k) {
            uint32_t pid = s->sorted[k];
            v3 velocity = V(0, 0, 0);
            m3 grad = mzero();
            REAL vgd = 0;
            if (s->enabled[pid] != 0) {
                v3 pt = s->pos[pid];
                v3 ref = vsub(vmul(assoc_cell_of(dx, pt), dx), pt);
                v3 w[3] = {kernel_eval_all(-ref.x / dx), kernel_eval_all(-ref.y / dx), kernel_eval_all(-ref.z / dx)};
                uint32_t a[3];
                assoc_in_block(dx, pt, a);
                for (int i = 0; i < 27; ++i) {
                    int sx = NBH_SHIFTS[i][0], sy = NBH_SHIFTS[i][1], sz = NBH_SHIFTS[i][2];
                    v3 cv = halo_vel(s, oct, (int)a[0] + sx, (int)a[1] + sy, (int)a[2] + sz);
                    v3 dpt = vadd(ref, vmul(V((REAL)sx, (REAL)sy, (REAL)sz), dx));
                    if (s->use_cpic) {
                        /* g2p.rs:206-235: an incompatible node gives its second velocity,
                         * projected by the closest body's boundary condition */
                        const node_t *nd = halo_node(s, oct, (int)a[0] + sx, (int)a[1] + sy, (int)a[2] + sz);
                        uint32_t naff = nd ? nd->cdf_aff : 0u, nclosest = nd ? nd->cdf_closest : NONE_U32;
                        if (!aff_compatible(s->cdf_aff[pid], naff)) {
                            cv = nd ? nd->mv_incompat : V(0, 0, 0);
                            if (nclosest != NONE_U32) {
                                const collider_t *c = &s->col[nclosest];
                                v3 cell_center = vadd(dpt, pt);
                                v3 bv = velocity_at_point(c, cell_center);
                                cv = vadd(bv, bc_project(c->bc_type, c->bc_friction * s->bfric[pid], vsub(cv, bv),
                                                         s->cdf_normal[pid]));
                            }
                        }
                    }
                    REAL weight = vget(w[0], sx) * vget(w[1], sy) * vget(w[2], sz);
                    velocity = vadd(velocity, vmul(cv, weight));
                    grad = madd(grad, mscale(mouter(cv, dpt), weight * inv_d));
                    vgd += weight * inv_d * vdot(cv, dpt);
                }
            }
            if (s->use_cpic) {
                /* g2p.rs:248-262: rigid velocity of every collider the particle has affinity with */
                v3 rv = V(0, 0, 0);
                if (s->enabled[pid] != 0)
                    for (uint32_t ic = 0; ic < 16 && ic < s->ncol; ++ic)
                        if (s->cdf_aff[pid] & (1u << ic)) rv = vadd(rv, velocity_at_point(&s->col[ic], s->pos[pid]));
                s->cdf_rigid_vel[pid] = rv;
            }
            s->aff[pid] = grad;
            s->vgd[pid] = vgd;
            s->vel[pid] = velocity;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Particle update: solver/particle_update.rs:60-201                         */
/* ------------------------------------------------------------------------ */

void orc_particle_update(scene_t *s) {
    const REAL dx = s->dx, dt = s->dt;
    const int64_t n = (int64_t)s->n;
#pragma omp parallel for schedule(static)
    for (int64_t pi = 0; pi < n; ++pi) {
        uint32_t p = (uint32_t)pi;
        uint32_t tag = s->tag[p];
        int fluid = tag == MODEL_FLUID;
        v3 v = s->vel[p];
        m3 F = s->F[p];
        v3 pos = s->pos[p];
        /* particle_update.rs:98-102: reproject a penetrating particle (the Cdf is
         * zero without CPIC, so this and the penalty below never trigger then) */
        const REAL sd = s->cdf_sd[p];
        if (sd < (REAL)-0.05 * dx) {
            v3 rv = s->cdf_rigid_vel[p];
            v = vadd(rv, bc_project(BC_SLIP, (REAL)0.0, vsub(v, rv), s->cdf_normal[p]));
        }
        REAL vl = vlen(v);
        if (vl > dx / dt) v = vdiv(vmul(vdiv(v, vl), dx), dt);
        v = vdiv(v, (REAL)1.0 + s->damping[p] * dt);
        if (s->fixed[p] != 0) v = V(0, 0, 0);
        v3 np = vadd(pos, vmul(v, dt));
        if (sd < (REAL)-0.05 * dx) { /* particle_update.rs:132-136 penalty impulse, PENALTY_COEFF = 1e3 */
            REAL corrected = fmax(sd, (REAL)-0.3 * dx);
            v = vadd(v, vmul(s->cdf_normal[p], dt * -corrected * (REAL)1.0e3));
        }
        m3 A = s->aff[p];
        if (!fluid) {
            F = madd(F, mm(mscale(A, dt), F));
        } else {
            REAL d0 = F.c0.x;
            REAL rate = s->vgd[p] * dt / (REAL)3.0;
            rate = rclamp(rate, (REAL)-0.1, (REAL)0.1);
            REAL nd = rclamp(d0 + rate * d0, (REAL)0.5, (REAL)2.0);
            F = mdiag(vsplat(nd));
        }
        m3 tau = model_update(tag, &s->words[(size_t)p * MODEL_WORDS], &F, A);
        REAL inv_d = (REAL)4.0 / (dx * dx);
        m3 aff = msub(mscale(A, s->mass[p]), mscale(tau, s->init_volume[p] * inv_d * dt));
        int nan = (np.x != np.x) || (np.y != np.y) || (np.z != np.z);
        if (!nan && mdet(F) > (REAL)0.0) {
            s->pos[p] = np;
            s->aff[p] = aff;
        } else {
            s->enabled[p] = 0;
            v = V(0, 0, 0);
            F = mident();
            s->aff[p] = mzero();
            s->mass[p] = 0;
        }
        s->vel[p] = v;
        s->F[p] = F;
    }
}

/* dynamics/body.rs Velocity::integrate + rigid_impulses.rs:66-140 for
 * one-way coupled (zero inverse mass) bodies: velocities are unchanged and
 * poses advance by the velocity. */
static void integrate_bodies(scene_t *s) {
    for (uint32_t i = 0; i < s->ncol; ++i) {
        collider_t *c = &s->col[i];
        v3 init_com = pose_apply(c->pose, c->local_com);
        v3 init_tra = c->pose.tra;
        v3 sa = vmul(c->angvel, s->dt);
        /* glam Quat::from_scaled_axis */
        REAL ang = vlen(sa);
        quat dq;
        if (ang == 0) { dq.x = 0; dq.y = 0; dq.z = 0; dq.w = 1; }
        else {
            v3 ax = vdiv(sa, ang);
            REAL sh = sin(ang * (REAL)0.5), ch = cos(ang * (REAL)0.5);
            dq.x = ax.x * sh; dq.y = ax.y * sh; dq.z = ax.z * sh; dq.w = ch;
        }
        v3 dl = vmul(c->linvel, s->dt);
        v3 nt = vadd(vadd(init_com, qrot(dq, vsub(init_tra, init_com))), dl);
        quat nr = qmul(dq, c->pose.rot);
        /* glam Quat::normalize multiplies by the reciprocal length */
        REAL rl = (REAL)1.0 / sqrt(nr.x * nr.x + nr.y * nr.y + nr.z * nr.z + nr.w * nr.w);
        nr.x *= rl; nr.y *= rl; nr.z *= rl; nr.w *= rl;
        c->pose.rot = nr;
        c->pose.tra = nt;
    }
}

/* rigid_impulses.rs:167-185 world mass properties (centre of mass). */
static void update_world_com(scene_t *s) {
    for (uint32_t i = 0; i < s->ncol; ++i) s->col[i].com = pose_apply(s->col[i].pose, s->col[i].local_com);
}

/* ------------------------------------------------------------------------ */
/* CPIC CDF passes for analytic colliders                                    */
/* ------------------------------------------------------------------------ */

/* solver/grid_update_cdf.rs:18-58 collide(): per node, every ball / cuboid /
 * capsule within 1.5 dx (or containing it) sets its affinity bit (and sign
 * bit when inside); the closest one by unsigned distance is kept.  Triangle
 * meshes reach the node CDF through rigid particles (orc_p2g_cdf). */
void orc_grid_update_cdf(scene_t *s) {
    const REAL dx = s->dx, cap = s->dx * (REAL)1.5;
    const int64_t nb = (int64_t)s->num_blocks;
#pragma omp parallel for schedule(static)
    for (int64_t bi = 0; bi < nb; ++bi) {
        const i3 vid = s->hdr[bi].vid;
        for (int t = 0; t < 64; ++t) {
            v3 point = vmul(V((REAL)(vid.x * 4 + (t & 3)), (REAL)(vid.y * 4 + ((t >> 2) & 3)), (REAL)(vid.z * 4 + (t >> 4))), dx);
            REAL dist = MAX_FLT;
            uint32_t affb = 0, closest = NONE_U32;
            for (uint32_t i = 0; i < s->ncol && i < 16; ++i) {
                const collider_t *c = &s->col[i];
                if (c->type == SHAPE_TRIMESH) continue;
                v3 local = pose_inv_apply(c->pose, point);
                proj_t pr;
                if (c->type == SHAPE_BALL) pr = ball_project_local(c->a[0], local);
                else if (c->type == SHAPE_CUBOID) pr = cuboid_project_local(V(c->a[0], c->a[1], c->a[2]), local);
                else if (c->type == SHAPE_CAPSULE)
                    pr = capsule_project_local(V(c->a[0], c->a[1], c->a[2]), V(c->b[0], c->b[1], c->b[2]), c->b[3], local);
                else { pr.point = local; pr.inside = 0; }
                pr.point = pose_apply(c->pose, pr.point);
                v3 dpt = vsub(pr.point, point);
                v3 ad = vabs(dpt);
                int within = ad.x <= cap && ad.y <= cap && ad.z <= cap;
                if (pr.inside || within) {
                    REAL d = vlen(dpt);
                    if (d < dist) { closest = i; dist = d; }
                    affb |= (pr.inside ? 0x00010001u : 0x00000001u) << i;
                }
            }
            node_t *nd = &s->nodes[(size_t)bi * 64 + t];
            nd->cdf_distance = dist;
            nd->cdf_aff = affb;
            nd->cdf_closest = closest;
        }
    }
}

/* solver/p2g_cdf.rs:52-259 gpu_p2g_cdf: every rigid particle listed in a
 * block projects the node positions of the block within its 3-cell range
 * (associated cell round(x / dx) - 1 to + 2) on its triangle (world
 * vertices = pose * local vertices, rigid_particle_update.rs:33-54); a
 * projection inside the face sets the collider's affinity bit (and the sign
 * bit for a node behind the face) and may lower the node distance (strict
 * <, list order = ascending particle order). */
void orc_p2g_cdf(scene_t *s) {
    const REAL dx = s->dx;
    const int64_t nb = (int64_t)s->num_blocks;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t bi = 0; bi < nb; ++bi) {
        const header_t *h = &s->hdr[bi];
        if (h->num_rigid == 0) continue;
        const i3 vid = h->vid;
        for (int t = 0; t < 64; ++t) {
            const i3 cell = {vid.x * 4 + (t & 3), vid.y * 4 + ((t >> 2) & 3), vid.z * 4 + (t >> 4)};
            const v3 cell_pos = vmul(V((REAL)cell.x, (REAL)cell.y, (REAL)cell.z), dx);
            node_t *nd = &s->nodes[(size_t)bi * 64 + t];
            for (uint32_t k = 0; k < h->num_rigid; ++k) {
                const uint32_t p = s->rp_sorted[h->first_rigid + k];
                const v3 ac = assoc_cell_of(dx, s->rp_world[p]);
                const int32_t sx = cell.x - r_to_i32(ac.x), sy = cell.y - r_to_i32(ac.y), sz = cell.z - r_to_i32(ac.z);
                if (sx < 0 || sx > 2 || sy < 0 || sy > 2 || sz < 0 || sz > 2) continue;
                const uint32_t cid = s->rp_col[p];
                const collider_t *c = &s->col[cid];
                const v3 *tv = &s->tri[3 * (size_t)s->rp_tri[p]];
                const v3 a = pose_apply(c->pose, tv[0]), b = pose_apply(c->pose, tv[1]), cc = pose_apply(c->pose, tv[2]);
                const v3 ap = vsub(cell_pos, a), bp = vsub(cell_pos, b), cp = vsub(cell_pos, cc);
                const v3 ab = vsub(b, a), acv = vsub(cc, a), bc = vsub(cc, b);
                const v3 n = vcross(ab, acv);
                const REAL nl = vlen(n);
                if (nl != 0 && vdot(vcross(ab, n), ap) <= 0 && vdot(vcross(bc, n), bp) <= 0 &&
                    vdot(vcross(acv, n), cp) >= 0) {
                    const REAL sd = vdot(n, ap) / nl;
                    const REAL d = fabs(sd);
                    nd->cdf_aff |= (sd < 0 ? 0x00010001u : 0x00000001u) << cid;
                    if (d < nd->cdf_distance) {
                        nd->cdf_distance = d;
                        nd->cdf_closest = cid;
                    }
                }
            }
        }
    }
}

/* Inverse and determinant of a 4x4 matrix m[row][col] from its 2x2 minors
 * (Laplace expansion along the first two rows). */
static REAL inv4(const REAL m[4][4], REAL out[4][4]) {
    REAL s0 = m[0][0] * m[1][1] - m[1][0] * m[0][1];
    REAL s1 = m[0][0] * m[1][2] - m[1][0] * m[0][2];
    REAL s2 = m[0][0] * m[1][3] - m[1][0] * m[0][3];
    REAL s3 = m[0][1] * m[1][2] - m[1][1] * m[0][2];
    REAL s4 = m[0][1] * m[1][3] - m[1][1] * m[0][3];
    REAL s5 = m[0][2] * m[1][3] - m[1][2] * m[0][3];
    REAL c5 = m[2][2] * m[3][3] - m[3][2] * m[2][3];
    REAL c4 = m[2][1] * m[3][3] - m[3][1] * m[2][3];
    REAL c3 = m[2][1] * m[3][2] - m[3][1] * m[2][2];
    REAL c2 = m[2][0] * m[3][3] - m[3][0] * m[2][3];
    REAL c1 = m[2][0] * m[3][2] - m[3][0] * m[2][2];
    REAL c0 = m[2][0] * m[3][1] - m[3][0] * m[2][1];
    REAL det = s0 * c5 - s1 * c4 + s2 * c3 + s3 * c2 - s4 * c1 + s5 * c0;
    REAL id = (REAL)1.0 / det;
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

double orc_inv4(const double *m16, double *out16) {
    REAL m[4][4], o[4][4];
    for (int i = 0; i < 16; ++i) m[i / 4][i % 4] = (REAL)m16[i];
    REAL d = inv4(m, o);
    for (int i = 0; i < 16; ++i) out16[i] = (double)o[i / 4][i % 4];
    return (double)d;
}

/* solver/g2p_cdf.rs:150-290 particle_g2p: the particle's affinity (the node
 * bits, with sign bits remembered from the previous step or, for a new
 * affinity, from the sign of the weighted node distances) and an MLS fit
 * of the signed distance field, distance = n . dpt + d, over the nodes that
 * share an affinity with it: normal = n / |n|, signed distance = d. */
void orc_g2p_cdf(scene_t *s) {
    const REAL dx = s->dx;
    const int64_t nb = (int64_t)s->num_blocks;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t bi = 0; bi < nb; ++bi) {
        const header_t *h = &s->hdr[bi];
        uint32_t oct[8];
        for (int o = 0; o < 8; ++o) oct[o] = find_header(s, i3add(h->vid, ASSOC_SHIFT[o]));
        for (uint32_t k = h->first_particle; k < h->first_particle + h->num_particles; ++k) {
            uint32_t pid = s->sorted[k];
            const uint32_t prev = s->cdf_aff[pid];
            v3 pt = s->pos[pid];
            v3 ref = vsub(vmul(assoc_cell_of(dx, pt), dx), pt);
            v3 w[3] = {kernel_eval_all(-ref.x / dx), kernel_eval_all(-ref.y / dx), kernel_eval_all(-ref.z / dx)};
            uint32_t a[3];
            assoc_in_block(dx, pt, a);
            uint32_t pa = 0;
            REAL sums[16];
            for (int ic = 0; ic < 16; ++ic) sums[ic] = 0;
            for (int i = 0; i < 27; ++i) {
                int sx = NBH_SHIFTS[i][0], sy = NBH_SHIFTS[i][1], sz = NBH_SHIFTS[i][2];
                const node_t *nd = halo_node(s, oct, (int)a[0] + sx, (int)a[1] + sy, (int)a[2] + sz);
                uint32_t naff = nd ? nd->cdf_aff : 0u;
                REAL ndist = nd ? nd->cdf_distance : MAX_FLT;
                pa |= naff & AFF_MASK;
                REAL weight = vget(w[0], sx) * vget(w[1], sy) * vget(w[2], sz);
                for (int ic = 0; ic < 16; ++ic) {
                    REAL compatible = (naff & (1u << ic)) ? (REAL)1.0 : (REAL)0.0;
                    REAL sign = ((naff >> AFF_SIGN_SHIFT) & (1u << ic)) ? (REAL)-1.0 : (REAL)1.0;
                    sums[ic] += compatible * weight * sign * ndist;
                }
            }
            for (int ic = 0; ic < 16; ++ic) {
                if (!(prev & (1u << ic))) {
                    if (sums[ic] < 0) pa |= 0x00010000u << ic;
                } else {
                    pa |= prev & (0x00010000u << ic);
                }
            }
            REAL q[4][4] = {{0}}, u[4] = {0, 0, 0, 0};
            for (int i = 0; i < 27; ++i) {
                int sx = NBH_SHIFTS[i][0], sy = NBH_SHIFTS[i][1], sz = NBH_SHIFTS[i][2];
                const node_t *nd = halo_node(s, oct, (int)a[0] + sx, (int)a[1] + sy, (int)a[2] + sz);
                uint32_t naff = nd ? nd->cdf_aff : 0u;
                REAL ndist = nd ? nd->cdf_distance : MAX_FLT;
                v3 dpt = vadd(ref, vmul(V((REAL)sx, (REAL)sy, (REAL)sz), dx));
                REAL weight = vget(w[0], sx) * vget(w[1], sy) * vget(w[2], sz);
                uint32_t combined = naff & pa & AFF_MASK;
                uint32_t sdiff = ((naff >> AFF_SIGN_SHIFT) ^ (pa >> AFF_SIGN_SHIFT)) & combined;
                REAL pv[4] = {dpt.x, dpt.y, dpt.z, (REAL)1.0};
                if (combined != 0) {
                    REAL dd = sdiff == 0 ? ndist : -ndist;
                    for (int r = 0; r < 4; ++r)
                        for (int c = 0; c < 4; ++c) q[r][c] += pv[r] * pv[c] * weight;
                    for (int r = 0; r < 4; ++r) u[r] += pv[r] * (weight * dd);
                }
            }
            REAL qi[4][4];
            REAL det = inv4(q, qi);
            if (det > (REAL)1.0e-8) {
                REAL r[4];
                for (int i = 0; i < 4; ++i) r[i] = qi[i][0] * u[0] + qi[i][1] * u[1] + qi[i][2] * u[2] + qi[i][3] * u[3];
                v3 nv = V(r[0], r[1], r[2]);
                REAL len = vlen(nv);
                s->cdf_normal[pid] = len > (REAL)1.0e-6 ? vdiv(nv, len) : V(0, 0, 0);
                s->cdf_sd[pid] = r[3];
                s->cdf_rigid_vel[pid] = V(0, 0, 0);
                s->cdf_aff[pid] = pa;
            } else {
                s->cdf_normal[pid] = V(0, 0, 0);
                s->cdf_sd[pid] = 0;
                s->cdf_rigid_vel[pid] = V(0, 0, 0);
                s->cdf_aff[pid] = 0;
            }
        }
    }
}

/* src_mpm/pipeline.rs:385-526 MpmPipeline::step; with CPIC, the node and
 * particle CDF passes run between the sort and P2G. */
int orc_step(scene_t *s) {
    update_world_com(s);
    if (s->use_cpic) {  /* pipeline.rs:393-405 rigid update */
        if (s->rp_dirty) build_rigid_particles(s);
        transform_rigid_particles(s);
    }
    orc_sort(s);
    if (s->use_cpic) {  /* pipeline.rs:433-460 */
        orc_grid_update_cdf(s);
        orc_p2g_cdf(s);
        orc_g2p_cdf(s);
    }
    orc_p2g(s);
    orc_grid_update(s);
    orc_g2p(s);
    orc_particle_update(s);
    integrate_bodies(s);
    return (int)s->status;
}

int orc_run(scene_t *s, uint32_t steps) {
    for (uint32_t i = 0; i < steps; ++i) orc_step(s);
    return (int)s->status;
}

/* ------------------------------------------------------------------------ */
/* Accessors for the parity tests                                            */
/* ------------------------------------------------------------------------ */

/* ------------------------------------------------------------------------ */
/* CFL timestep bound: solver/timestep_bound.rs:59-115 (per particle, min),   */
/* models/default.rs:268-343 (model sound speed), models/utils.rs:157-175.    */
/* ------------------------------------------------------------------------ */

/* utils.rs:157-175 ElasticitySoundSpeedTimestepBound::timestep_bound */
static REAL sound_speed_bound(REAL alpha, REAL bulk, REAL shear, REAL density0, REAL def_grad_det, v3 vel,
                              REAL cell_width) {
    REAL curr_density = density0 / fmax(def_grad_det, (REAL)1.0e-6);
    REAL sound_speed = sqrt((bulk + shear * (REAL)4.0 / (REAL)3.0) / curr_density);
    REAL max_speed = fmax(vlen(vel), sound_speed);
    return alpha * cell_width / max_speed;
}

/* linear_elasticity.rs:58-80 / neo_hookean_elasticity.rs:43-65 on words w[o..o+3) = lambda, mu, cfl */
static REAL elastic_bound(const REAL *w, int o, REAL hardening, REAL density0, REAL jdet, v3 vel, REAL cw) {
    REAL lambda = w[o], mu = w[o + 1], cfl = w[o + 2];
    REAL bulk = lambda + (REAL)2.0 * mu / (REAL)3.0; /* utils.rs:34-36 */
    REAL shear = mu;                                 /* utils.rs:28-30 */
    return sound_speed_bound(cfl, bulk * hardening, shear * hardening, density0, jdet, vel, cw);
}

/* The bound in the reference's fixed-point form: (dt * 1e12) as u32, the
 * minimum over enabled particles (0xFFFFFFFF when none). */
uint32_t orc_timestep_bound_bits(const scene_t *s) {
    uint32_t best = 0xFFFFFFFFu;
    const REAL cw = s->dx;
    for (uint32_t p = 0; p < s->n; ++p) {
        if (s->enabled[p] == 0) continue;
        const REAL *w = &s->words[(size_t)p * MODEL_WORDS];
        REAL density0 = s->mass[p] / s->init_volume[p];
        REAL jdet = mdet(s->F[p]);
        v3 vel = s->vel[p];
        REAL dt;
        switch (s->tag[p]) {
        case MODEL_ELASTIC_LINEAR:
        case MODEL_ELASTIC_NEO_HOOKEAN: dt = elastic_bound(w, 0, (REAL)1.0, density0, jdet, vel, cw); break;
        case MODEL_SAND_LINEAR:
        case MODEL_SAND_NEO_HOOKEAN: dt = elastic_bound(w, 10, (REAL)1.0, density0, jdet, vel, cw); break;
        case MODEL_FLUID: /* fluid.rs:88-108: bulk modulus * gamma, no shear; words k, gamma, mu, cfl, t */
            dt = sound_speed_bound(w[3], w[0] * w[1], (REAL)0.0, density0, jdet, vel, cw);
            break;
        case MODEL_SNOW: { /* snow.rs:77-79 hardening = exp(h (1 - plastic_det)); elastic words 4..6 */
            REAL hard = exp(w[3] * ((REAL)1.0 - w[0]));
            dt = elastic_bound(w, 4, hard, density0, jdet, vel, cw);
            break;
        }
        default: dt = (REAL)0.0; break;
        }
        m3 A = s->aff[p];
        REAL na2 = vdot(A.c0, A.c0) + vdot(A.c1, A.c1) + vdot(A.c2, A.c2);
        REAL d = (cw * cw) / (REAL)4.0;
        REAL norm_b = d * sqrt(na2) / s->mass[p];
        REAL apic_v = norm_b * (REAL)6.0 * sqrt((REAL)3.0) / cw;
        REAL v = vlen(vel) + apic_v;
        dt = fmin(dt, cw / v);
        /* Rust `as u32`: truncation, saturating, NaN -> 0 */
        REAL scaled = dt * (REAL)1.0e12;
        uint32_t c = scaled != scaled ? 0u : (scaled >= (REAL)4294967295.0 ? 0xFFFFFFFFu
                                                : (scaled <= 0 ? 0u : (uint32_t)scaled));
        if (c < best) best = c;
    }
    return best;
}

uint32_t orc_num_blocks(const scene_t *s) { return s->num_blocks; }
uint32_t orc_status(const scene_t *s) { return s->status; }
uint32_t orc_capacity(const scene_t *s) { return s->capacity; }

/* Per block (header order): vid[3], first, num, num_extras, cursors[10], nbh[7] = 23 int32. */
void orc_get_headers(const scene_t *s, int32_t *out) {
    for (uint32_t b = 0; b < s->num_blocks; ++b) {
        const header_t *h = &s->hdr[b];
        int32_t *o = out + 23 * (size_t)b;
        o[0] = h->vid.x; o[1] = h->vid.y; o[2] = h->vid.z;
        o[3] = (int32_t)h->first_particle; o[4] = (int32_t)h->num_particles; o[5] = (int32_t)h->num_particles_with_extras;
        for (int k = 0; k < NUM_BUCKETS; ++k) o[6 + k] = (int32_t)h->cursors[k];
        for (int k = 0; k < NUM_NBH; ++k) o[16 + k] = (int32_t)h->nbh[k];
    }
}

uint32_t orc_sorted_len(const scene_t *s) {
    if (s->num_blocks == 0) return 0;
    const header_t *h = &s->hdr[s->num_blocks - 1];
    return h->first_particle + h->num_particles_with_extras;
}

void orc_get_sorted(const scene_t *s, uint32_t *out) {
    uint32_t len = orc_sorted_len(s);
    memcpy(out, s->sorted, (size_t)len * sizeof(uint32_t));
}

/* Nodes of all active blocks, header order, 8 floats per node:
 * mv.xyz, mass, mv_incompat.xyz, mass_incompat. */
void orc_get_nodes(const scene_t *s, float *out) {
    for (size_t i = 0; i < (size_t)s->num_blocks * 64; ++i) {
        const node_t *nd = &s->nodes[i];
        float *o = out + 8 * i;
        o[0] = (float)nd->mv.x; o[1] = (float)nd->mv.y; o[2] = (float)nd->mv.z; o[3] = (float)nd->mass;
        o[4] = (float)nd->mv_incompat.x; o[5] = (float)nd->mv_incompat.y; o[6] = (float)nd->mv_incompat.z;
        o[7] = (float)nd->mass_incompat;
    }
}

/* ------------------------------------------------------------------------ */
/* Stand-alone pieces exposed for known-answer tests                         */
/* ------------------------------------------------------------------------ */

uint32_t orc_pack_key(int32_t x, int32_t y, int32_t z) { i3 b = {x, y, z}; return pack_key(b); }
uint32_t orc_hash(uint32_t k) { return hash_key(k); }
double orc_kernel_eval(double x) { return (double)kernel_eval((REAL)x); }
void orc_kernel_eval_all(double x, double *out3) {
    v3 r = kernel_eval_all((REAL)x);
    out3[0] = (double)r.x; out3[1] = (double)r.y; out3[2] = (double)r.z;
}
void orc_block_of_point(double dx, const float *pt, int32_t *out3, uint32_t *assoc3) {
    v3 p = V(pt[0], pt[1], pt[2]);
    i3 b = block_of_point((REAL)dx, p);
    out3[0] = b.x; out3[1] = b.y; out3[2] = b.z;
    assoc_in_block((REAL)dx, p, assoc3);
}
/* tau for one particle: F and velocity gradient column-major; words = 24 f32 bits; the
 * updated F and model words are written back. */
void orc_model_update(uint32_t tag, uint32_t *words, float *F, const float *vel_grad, float *tau) {
    REAL w[MODEL_WORDS];
    for (int k = 0; k < MODEL_WORDS; ++k) w[k] = bits2f(words[k]);
    m3 f = load_m3(F);
    m3 t = model_update(tag, w, &f, load_m3(vel_grad));
    store_m3(F, f);
    store_m3(tau, t);
    for (int k = 0; k < MODEL_WORDS; ++k) words[k] = f2bits((float)w[k]);
}
void orc_svd(const float *F, float *u, float *sig, float *vt) {
    svd3 d = svd(load_m3(F));
    store_m3(u, d.u);
    sig[0] = (float)d.s.x; sig[1] = (float)d.s.y; sig[2] = (float)d.s.z;
    store_m3(vt, d.vt);
}
/* Projection of a world point on collider i: out = point xyz, inside flag. */
int orc_project_point(const scene_t *s, uint32_t i, const float *pt, float *out3) {
    const collider_t *c = &s->col[i];
    v3 p = V(pt[0], pt[1], pt[2]);
    proj_t pr;
    int valid = 1;
    if (c->type == SHAPE_TRIMESH) {
        v3 local = pose_inv_apply(c->pose, p);
        pr = trimesh_project(s, c, local, MAX_FLT, &valid);
    } else {
        v3 local = pose_inv_apply(c->pose, p);
        if (c->type == SHAPE_BALL) pr = ball_project_local(c->a[0], local);
        else if (c->type == SHAPE_CUBOID) pr = cuboid_project_local(V(c->a[0], c->a[1], c->a[2]), local);
        else pr = capsule_project_local(V(c->a[0], c->a[1], c->a[2]), V(c->b[0], c->b[1], c->b[2]), c->b[3], local);
    }
    pr.point = pose_apply(c->pose, pr.point);
    out3[0] = (float)pr.point.x; out3[1] = (float)pr.point.y; out3[2] = (float)pr.point.z;
    return valid ? pr.inside : -1;
}
void orc_bc_project(uint32_t ty, float friction, const float *vel, const float *n, float *out3) {
    v3 r = bc_project(ty, friction, V(vel[0], vel[1], vel[2]), V(n[0], n[1], n[2]));
    out3[0] = (float)r.x; out3[1] = (float)r.y; out3[2] = (float)r.z;
}
/* src_rbd/utils/prefix_sum.rs:112-136 CPU semantics: inclusive wrapping sum, shift right, leading 0. */
void orc_prefix_sum(uint32_t *v, uint32_t len) {
    if (len == 0) return;
    for (uint32_t i = 0; i + 1 < len; ++i) v[i + 1] = v[i + 1] + v[i];
    for (uint32_t i = len - 1; i >= 1; --i) v[i] = v[i - 1];
    v[0] = 0;
}

/* ------------------------------------------------------------------------ */
/* Trimesh projection (brute force over the collider's triangles)            */
/* ------------------------------------------------------------------------ */

/* Closest point on triangle (a, b, c) to p, with the feature it lies on:
 * feature 0 = vertex (id 0..2), 1 = edge (id 0 = ab, 1 = ac... see below),
 * 2 = face.  Edge ids follow the reference's pseudo-normal table
 * (trimesh.rs:129-140): 0 = ab, 1 = bc, 2 = ca. */
typedef struct { v3 point; int feature; int id; } tri_proj_t;

static tri_proj_t triangle_closest(v3 a, v3 b, v3 c, v3 p) {
    /* Ericson, Real-Time Collision Detection, 5.1.5 (Voronoi regions). */
    tri_proj_t r;
    v3 ab = vsub(b, a), ac = vsub(c, a), ap = vsub(p, a);
    REAL d1 = vdot(ab, ap), d2 = vdot(ac, ap);
    if (d1 <= 0 && d2 <= 0) { r.point = a; r.feature = 0; r.id = 0; return r; }
    v3 bp = vsub(p, b);
    REAL d3 = vdot(ab, bp), d4 = vdot(ac, bp);
    if (d3 >= 0 && d4 <= d3) { r.point = b; r.feature = 0; r.id = 1; return r; }
    REAL vc = d1 * d4 - d3 * d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0) {
        REAL v = d1 / (d1 - d3);
        r.point = vadd(a, vmul(ab, v)); r.feature = 1; r.id = 0; return r;
    }
    v3 cp = vsub(p, c);
    REAL d5 = vdot(ab, cp), d6 = vdot(ac, cp);
    if (d6 >= 0 && d5 <= d6) { r.point = c; r.feature = 0; r.id = 2; return r; }
    REAL vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) {
        REAL w = d2 / (d2 - d6);
        r.point = vadd(a, vmul(ac, w)); r.feature = 1; r.id = 2; return r;
    }
    REAL va = d3 * d6 - d5 * d4;
    if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
        REAL w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        r.point = vadd(b, vmul(vsub(c, b), w)); r.feature = 1; r.id = 1; return r;
    }
    REAL denom = (REAL)1.0 / (va + vb + vc);
    REAL v = vb * denom, w = vc * denom;
    r.point = vadd(a, vadd(vmul(ab, v), vmul(ac, w)));
    r.feature = 2; r.id = 0;
    return r;
}

/* trimesh.rs:155-207: closest triangle within max_dist; inside test with the
 * angle-weighted pseudo-normal of the closest feature (Baerentzen & Aanaes
 * 2005), computed here from the triangle soup instead of the precomputed
 * per-vertex/per-edge tables the reference uploads. */
static proj_t trimesh_project(const scene_t *s, const collider_t *c, v3 pt, REAL max_dist, int *valid) {
    REAL best = max_dist;
    int found = 0;
    tri_proj_t bp = {pt, 2, 0};
    uint32_t best_t = 0;
    for (uint32_t t = c->tri_first; t < c->tri_first + c->tri_count; ++t) {
        v3 a = s->tri[3 * t], b = s->tri[3 * t + 1], cc = s->tri[3 * t + 2];
        tri_proj_t pr = triangle_closest(a, b, cc, pt);
        REAL d = vlen(vsub(pr.point, pt));
        if (d <= best) { best = d; bp = pr; best_t = t; found = 1; }
    }
    proj_t out;
    if (!found) { *valid = 0; out.point = V(0, 0, 0); out.inside = 0; return out; }
    *valid = 1;
    v3 a = s->tri[3 * best_t], b = s->tri[3 * best_t + 1], cc = s->tri[3 * best_t + 2];
    v3 pn;
    if (bp.feature == 2) {
        pn = vcross(vsub(b, a), vsub(cc, a));
    } else {
        /* pseudo-normal of a vertex / edge: angle-weighted / summed face
         * normals of every triangle of this mesh sharing that feature. */
        v3 fa = bp.feature == 0 ? (bp.id == 0 ? a : (bp.id == 1 ? b : cc)) : V(0, 0, 0);
        v3 e0 = a, e1 = b;
        if (bp.feature == 1) {
            if (bp.id == 0) { e0 = a; e1 = b; } else if (bp.id == 1) { e0 = b; e1 = cc; } else { e0 = cc; e1 = a; }
        }
        pn = V(0, 0, 0);
        for (uint32_t t = c->tri_first; t < c->tri_first + c->tri_count; ++t) {
            v3 q[3] = {s->tri[3 * t], s->tri[3 * t + 1], s->tri[3 * t + 2]};
            v3 fn = vcross(vsub(q[1], q[0]), vsub(q[2], q[0]));
            REAL fl = vlen(fn);
            if (fl == 0) continue;
            fn = vdiv(fn, fl);
            for (int k = 0; k < 3; ++k) {
                if (bp.feature == 0) {
                    if (q[k].x == fa.x && q[k].y == fa.y && q[k].z == fa.z) {
                        v3 u = vsub(q[(k + 1) % 3], q[k]), w = vsub(q[(k + 2) % 3], q[k]);
                        REAL cosang = vdot(u, w) / (vlen(u) * vlen(w));
                        cosang = rclamp(cosang, (REAL)-1.0, (REAL)1.0);
                        pn = vadd(pn, vmul(fn, acos(cosang)));
                    }
                } else {
                    v3 q0 = q[k], q1 = q[(k + 1) % 3];
                    int same = (q0.x == e0.x && q0.y == e0.y && q0.z == e0.z && q1.x == e1.x && q1.y == e1.y && q1.z == e1.z) ||
                               (q0.x == e1.x && q0.y == e1.y && q0.z == e1.z && q1.x == e0.x && q1.y == e0.y && q1.z == e0.z);
                    if (same) pn = vadd(pn, fn);
                }
            }
        }
    }
    out.point = bp.point;
    out.inside = vdot(pn, vsub(pt, bp.point)) <= 0;
    return out;
}

/* ------------------------------------------------------------------------ */
/* Render data: src_mpm_shaders/solver/prep_readback.rs (3D)                 */
/* ------------------------------------------------------------------------ */

/* GpuReadbackData::DEFAULT_GROUP_COLORS (src_mpm/solver/prep_readback.rs). */
static const float DEFAULT_PALETTE[6][4] = {
    {124.0f / 255.0f, 144.0f / 255.0f, 1.0f, 1.0f},           {8.0f / 255.0f, 144.0f / 255.0f, 1.0f, 1.0f},
    {124.0f / 255.0f, 7.0f / 255.0f, 1.0f, 1.0f},             {124.0f / 255.0f, 144.0f / 255.0f, 7.0f / 255.0f, 1.0f},
    {200.0f / 255.0f, 37.0f / 255.0f, 1.0f, 1.0f},            {124.0f / 255.0f, 230.0f / 255.0f, 25.0f / 255.0f, 1.0f}};

static inline void put4(float *o, float a, float b, float c, float d) { o[0] = a; o[1] = b; o[2] = c; o[3] = d; }

/* One ReadbackData record, 24 floats: color, deformation as a column-major
 * 4x4 (Mat4::from_mat3), position, padding. */
static void readback_record(float *o, const float color[4], m3 def, v3 pos) {
    put4(o, color[0], color[1], color[2], color[3]);
    put4(o + 4, (float)def.c0.x, (float)def.c0.y, (float)def.c0.z, 0.0f);
    put4(o + 8, (float)def.c1.x, (float)def.c1.y, (float)def.c1.z, 0.0f);
    put4(o + 12, (float)def.c2.x, (float)def.c2.y, (float)def.c2.z, 0.0f);
    put4(o + 16, 0.0f, 0.0f, 0.0f, 1.0f);
    put4(o + 20, (float)pos.x, (float)pos.y, (float)pos.z, 0.0f);
}

/* prep_readback.rs:241-295 gpu_prep_readback: per particle (id order) its
 * color for the render mode (compute_color, :176-237), its deformation
 * diag(2 r) * clamp(F, -4, 4) (compute_deformation, :111-123) and position.
 * `palette` holds `num_groups` rgba colors (NULL: the default palette). */
void orc_prep_readback(const scene_t *s, uint32_t mode, const float *palette, uint32_t num_groups, float *out24) {
    if (!palette || num_groups == 0) { palette = &DEFAULT_PALETTE[0][0]; num_groups = 6; }
    for (uint32_t i = 0; i < s->n; ++i) {
        const float *bc = palette + 4 * (size_t)(s->group_id[i] % num_groups);
        float col[4] = {bc[0], bc[1], bc[2], bc[3]};  /* every mode keeps the base alpha */
        if (mode == 2) { /* velocity */
            v3 c = vadd(vmul(vmul(vabs(s->vel[i]), s->dt), (REAL)100.0), vsplat((REAL)0.2));
            col[0] = (float)c.x; col[1] = (float)c.y; col[2] = (float)c.z;
        } else if (mode == 1) { /* volume */
            svd3 d = svd(s->F[i]);
            v3 c = vadd(vdiv(vsub(vsplat((REAL)1.0), d.s), (REAL)0.005), vsplat((REAL)0.2));
            col[0] = (float)c.x; col[1] = (float)c.y; col[2] = (float)c.z;
        } else if (mode == 3) { /* phase */
            const REAL ph = s->phase[i];
            col[0] = 0.0f; col[1] = (float)((REAL)0.4 * ph); col[2] = (float)((REAL)0.4 * ((REAL)1.0 - ph));
        } else if (mode == 4) { /* cdf normals */
            v3 nrm = s->cdf_normal[i];
            if (nrm.x == 0 && nrm.y == 0 && nrm.z == 0) { col[0] = col[1] = col[2] = 0.0f; }
            else {
                v3 c = vmul(vadd(nrm, vsplat((REAL)1.0)), (REAL)0.5);
                col[0] = (float)c.x; col[1] = (float)c.y; col[2] = (float)c.z;
            }
        } else if (mode == 5) { /* cdf distances */
            REAL d = s->cdf_sd[i] / (s->dx * (REAL)1.5);
            if (d > 0) { col[0] = 0.0f; col[1] = (float)fabs(d); col[2] = 0.0f; }
            else { col[0] = (float)fabs(d); col[1] = 0.0f; col[2] = 0.0f; }
        } else if (mode == 6) { /* cdf signs */
            uint32_t a = s->cdf_aff[i];
            uint32_t both = (a >> 16) & (a & 0x0000FFFFu);
            col[0] = (a != 0 && both != 0) ? 1.0f : 0.0f;
            col[1] = (a != 0 && both == 0) ? 1.0f : 0.0f;
            col[2] = 0.0f;
        }
        if (!s->enabled[i]) put4(col, 1.0f, 0.0f, 0.0f, 1.0f);
        const REAL r2 = (REAL)s->init_radius[i] * (REAL)2.0;
        m3 cl = M(vclamp(s->F[i].c0, -4, 4), vclamp(s->F[i].c1, -4, 4), vclamp(s->F[i].c2, -4, 4));
        m3 def = mm(mdiag(vsplat(r2)), cl);
        readback_record(out24 + 24 * (size_t)i, col, def, s->pos[i]);
    }
}

/* prep_readback.rs:420-469 gpu_prep_readback_rigid: per rigid particle its
 * base color (`colors`, 4 per particle; NULL: the palette cycled over the
 * particles, GpuReadbackData::new), the deformation diag(0.4 dx) and its
 * world position. */
void orc_prep_readback_rigid(scene_t *s, const float *colors, const float *palette, uint32_t num_groups,
                             float *out24) {
    if (s->rp_dirty) build_rigid_particles(s);
    if (!palette || num_groups == 0) { palette = &DEFAULT_PALETTE[0][0]; num_groups = 6; }
    const REAL scale = s->dx * (REAL)0.4;
    for (uint32_t i = 0; i < s->nrp; ++i) {
        const float *c = colors ? colors + 4 * (size_t)i : palette + 4 * (size_t)(i % num_groups);
        readback_record(out24 + 24 * (size_t)i, c, mdiag(vsplat(scale)), s->rp_world[i]);
    }
}
