// Memory layout of one MPM state in HBM (shared by the host library and the kernels).
//
// Particles are stored as two 16-byte-aligned records so that a particle
// gathered through the sorted index costs whole 32-byte sectors (in the fast
// mode the records are kept in the previous step's sorted order, double
// buffered, with the particle id of each slot alongside):
//   PKin (80 B): x, mass | v, flags | C columns (c0.w = vel_grad_det)
//   PDef (48 B): F columns | (f0.w = V0, f1.w = damping, f2.w = material id)
// plus, for plastic models only, a float4 of model state words.
// The grid is a hash of 4x4x4-node blocks: packed block keys, per-block
// headers (struct-of-arrays), 64 float4 nodes per block (momentum + mass,
// then velocity + mass after the grid update).
#pragma once

#include <cstdint>

namespace nxm {

constexpr uint32_t NONE = 0xFFFFFFFFu;
constexpr int NUM_PRIMARY_BUCKETS = 4;
constexpr int NUM_EXTRA_BUCKETS = 6;
constexpr int NUM_BUCKETS = 10;
constexpr int NUM_NBH = 7;
constexpr int MODEL_WORDS = 24;
constexpr float MAX_FLT = 1.0e18f;  // nexus_rbd_shaders::MAX_FLT
constexpr int MAX_COLLIDERS = 16;   // solver/boundary_condition.rs:132

enum : uint32_t {
    MODEL_ELASTIC_LINEAR = 0,
    MODEL_ELASTIC_NEO_HOOKEAN = 1,
    MODEL_SAND_LINEAR = 2,
    MODEL_SAND_NEO_HOOKEAN = 3,
    MODEL_FLUID = 4,
    MODEL_SNOW = 5,
};

enum : uint32_t { BC_STICK = 0, BC_SLIP = 1, BC_SEPARATE = 2, BC_NON_REFLECTING = 3 };
enum : uint32_t { SHAPE_BALL = 0, SHAPE_CUBOID = 1, SHAPE_CAPSULE = 2, SHAPE_TRIMESH = 6 };

// Particle flag bits (PKin.flags as u32 bits).
enum : uint32_t { PFLAG_ENABLED = 1u, PFLAG_FIXED = 2u };

// Device status bits (sticky until read by the host).
enum : uint32_t {
    STATUS_HASH_FULL = 1u,        // a block could not be inserted into the hash
    STATUS_BLOCK_CAPACITY = 2u,   // more active blocks than the grid capacity
    STATUS_MISSING_BLOCK = 4u,    // a particle's block was not found (follows 1 or 2)
    STATUS_SORT_CAPACITY = 8u,    // sorted-id list longer than its buffer
    STATUS_COPY_TIMEOUT = 16u,    // a bulk copy did not complete within its wait limit
};

struct alignas(16) PKin {
    float x, y, z, mass;
    float vx, vy, vz, flags;     // flags: PFLAG_* as u32 bits
    float c00, c10, c20, vgd;    // C column 0; w = vel_grad_det
    float c01, c11, c21, pad1;   // C column 1
    float c02, c12, c22, pad2;   // C column 2
};
static_assert(sizeof(PKin) == 80, "PKin layout");

struct alignas(16) PDef {
    float f00, f10, f20, init_volume;
    float f01, f11, f21, damping;
    float f02, f12, f22, material;  // material index (u32 bits)
};
static_assert(sizeof(PDef) == 48, "PDef layout");

// One deduplicated material: tag + the 24 model words as floats.  State
// words (Drucker-Prager words 0..2, snow word 0) live per particle.
struct alignas(16) Material {
    uint32_t tag;
    uint32_t has_state;  // 1 if the model mutates per-particle state words
    uint32_t pad[2];
    float w[MODEL_WORDS];
};
static_assert(sizeof(Material) == 112, "Material layout");

// Device form of a collider.
struct alignas(16) DevCollider {
    float a[4], b[4], c[4];
    float rot[4];   // quaternion x, y, z, w
    float tra[4];
    float linvel[4];
    float angvel[4];
    float local_com[4];
    float com[4];   // world centre of mass (refreshed at the start of a step)
    uint32_t type, bc_type, tri_first, tri_count;
    float bc_friction;
    uint32_t bvh_first, bvh_count;  // trimesh: its BVH nodes [bvh_first, bvh_first + bvh_count)
    uint32_t scene;                 // batched scenes: the scene owning it (NONE otherwise)
};
static_assert(sizeof(DevCollider) == 176, "DevCollider layout");

// One triangle of a trimesh collider (local frame of the mesh), with the
// pseudo-normals of its features for the inside test (Baerentzen & Aanaes
// 2005): pn[0..2] vertices a, b, c (angle-weighted), pn[3..5] edges ab, bc,
// ca (sum of the unit normals of the faces sharing the edge), pn[6] face
// (ab x ac, unnormalised).
struct alignas(16) DevTri {
    float v[3][4];
    float pn[7][4];
};
static_assert(sizeof(DevTri) == 160, "DevTri layout");

// Node of a stackless BVH in depth-first order.  Internal: `entry` = first
// child, `exit` = the node after this subtree.  Leaf: `entry` = kBvhLeaf |
// triangle index (into the state's triangle array).
constexpr uint32_t kBvhLeaf = 0x80000000u;
struct alignas(16) DevBvhNode {
    float mn[3];
    uint32_t entry;
    float mx[3];
    uint32_t exit;
};
static_assert(sizeof(DevBvhNode) == 32, "DevBvhNode layout");

// Per-step parameters read by every kernel from device memory (so a captured
// CUDA graph stays valid when they change).
struct alignas(16) Params {
    float gravity[3];
    float dt;
    float dx;
    float inv_dx;
    uint32_t n;              // particles
    uint32_t ncol;           // colliders
    uint32_t block_capacity; // headers / node blocks
    uint32_t hash_capacity;  // slots, power of two
    uint32_t sorted_capacity;
    uint32_t use_cpic;
    // Batched scenes (scene_blocks != 0): scene s owns the block-key region of
    // cell c(s) = (s mod cells[0], (s / cells[0]) mod cells[1], ...) + cmin, a
    // cube of scene_blocks blocks per axis.  Its particles keep scene-local
    // positions; a local block coordinate b in [-margin, scene_blocks - margin)
    // has the key of b + c(s) * scene_blocks.
    uint32_t scene_blocks;
    int32_t scene_margin;
    int32_t scene_cmin[3];
    uint32_t scene_cells[3];
    // the fast G2P takes one block per unit (instead of runs of the sorted
    // list) below this many particles per primary block on average (tuned)
    uint32_t range_min_fill;
    uint32_t pad[3];
};
static_assert(sizeof(Params) == 96, "Params layout");

// Device counters (reset each step by the sort).
struct alignas(16) Counters {
    uint32_t num_primary;   // blocks inserted by the primary pass
    uint32_t num_extra;     // blocks inserted by the neighbour pass
    uint32_t num_blocks;    // num_primary + num_extra (written by the scan)
    uint32_t sorted_len;    // total sorted ids, extras included
    uint32_t status;        // STATUS_* bits
    uint32_t codes_valid;   // 1 when pcode holds the block key of every particle's current position
    uint32_t unsorted;      // particles without a block this step, placed after the sorted ones
                            // by the reordering G2P
    uint32_t dt_bound;      // CFL bound, (dt * 1e12) as u32 (written by the timestep-bound query)
    uint32_t rigid_len;     // CPIC: entries of the block-sorted rigid-particle list
    uint32_t pad[3];
};
static_assert(sizeof(Counters) == 48, "Counters layout");

// CPIC rigid particle (a surface sample of a trimesh collider): position and
// a packed word, triangle index into the state's triangle array in the low
// kRigidTriBits bits, owning collider above them.
constexpr uint32_t kRigidTriBits = 28;
constexpr uint32_t kRigidTriMask = (1u << kRigidTriBits) - 1u;

}  // namespace nxm
