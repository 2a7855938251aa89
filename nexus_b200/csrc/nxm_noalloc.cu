// nxm_sort_blocks_noalloc: the block activation + particle sort for callers
// that cannot allocate device memory.
//
// Some callers of this library may not allocate GPU memory at all: a host
// program (a game engine, a simulation service) that reserves all of its
// device memory once at start-up and forbids allocations inside its frame
// loop, so that a frame can neither fail for lack of memory nor stall while
// the allocator synchronizes the device; or a plugin that runs inside such a
// program and is handed device buffers but no allocator.  This entry point
// runs the same sort kernels as nxm_step's sort, but keeps all of its grid
// tables (hash, block headers, bucket cursors, scan tiles, counters) in one
// file-scope `static __device__` array instead of state-owned allocations; the
// caller passes the particle positions and the output buffers.  It calls no
// cudaMalloc, cudaFree or other allocating routine.
//
// The array holds at most kNoallocMaxBlocks active blocks (about 1.9 MB, kept
// by every GPU that loads this library until the process exits).  In host
// code the array's name is not a device address: its address is looked up
// once per device (cudaGetSymbolAddress, return code checked) by the first
// call made with that device current, and kept for the life of the process,
// so the library must not be used across a cudaDeviceReset of that device.
// Every call shares the array: calls whose GPU work overlaps (different
// streams, or concurrent host threads) race on it and must be serialized by
// the caller.  A call waits for its stream before returning.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "../../include/nexus_mpm.h"
#include "nxm_kernels.h"
#include "nxm_layout.h"

using namespace nxm;

namespace {

constexpr uint32_t kNoallocMaxBlocks = NXM_NOALLOC_MAX_BLOCKS;
constexpr uint32_t kNoallocHash = 2u * kNoallocMaxBlocks;
constexpr uint32_t kNoallocTiles = kNoallocMaxBlocks / kScanTile + 2u;

// Byte offsets of each table inside the scratch array (all 256-byte aligned).
constexpr size_t align256(size_t v) { return (v + 255u) & ~size_t(255u); }
constexpr size_t kOffParams = 0;
constexpr size_t kOffCounters = align256(kOffParams + sizeof(Params));
constexpr size_t kOffHkey = align256(kOffCounters + sizeof(Counters));
constexpr size_t kOffHval = align256(kOffHkey + 4ull * kNoallocHash);
constexpr size_t kOffBvid = align256(kOffHval + 4ull * kNoallocHash);
constexpr size_t kOffFirst = align256(kOffBvid + 16ull * kNoallocMaxBlocks);
constexpr size_t kOffNprim = align256(kOffFirst + 4ull * kNoallocMaxBlocks);
constexpr size_t kOffNwx = align256(kOffNprim + 4ull * kNoallocMaxBlocks);
constexpr size_t kOffScanTmp = align256(kOffNwx + 4ull * kNoallocMaxBlocks);
constexpr size_t kOffCursors = align256(kOffScanTmp + 4ull * kNoallocMaxBlocks);
constexpr size_t kOffNbh = align256(kOffCursors + 4ull * NUM_BUCKETS * kNoallocMaxBlocks);
constexpr size_t kOffTiles = align256(kOffNbh + 4ull * NUM_NBH * kNoallocMaxBlocks);
constexpr size_t kScratchBytes = align256(kOffTiles + 4ull * kNoallocTiles);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of g_noalloc_scratch per device (host code cannot use the
// symbol itself as a device pointer).
constexpr int kMaxDevices = 64;
unsigned char* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

int scratch_for_current_device(unsigned char** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        (void)cudaGetLastError();
        return NXM_E_NO_DEVICE;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            (void)cudaGetLastError();
            return NXM_E_CUDA;
        }
        g_scratch_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_addr[dev];
    return NXM_OK;
}

// Writes this call's parameters and clears the counters (status included).
__global__ void k_noalloc_begin(Params prm, Params* params, Counters* counters) {
    if (threadIdx.x == 0) {
        *params = prm;
        Counters c{};
        *counters = c;
    }
}

// Copies the block table out: virtual id + key, first primary, primary count.
__global__ void k_noalloc_export(const int4* bvid, const uint32_t* first, const uint32_t* nprim,
                                 const Counters* counters, int4* out_vid, uint2* out_range, uint32_t max_blocks) {
    const uint32_t nb = min(counters->num_blocks, max_blocks);
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        out_vid[b] = bvid[b];
        out_range[b] = make_uint2(first[b], nprim[b]);
    }
}

}  // namespace

extern "C" int nxm_sort_blocks_noalloc(const float* positions, uint32_t n, float cell_width, uint32_t* sorted_ids,
                                       int32_t* block_vids, uint32_t* block_ranges, uint32_t max_blocks,
                                       uint32_t* num_blocks, void* stream) {
    if (!positions || !sorted_ids || !block_vids || !block_ranges || !num_blocks) return NXM_E_INVALID;
    if ((reinterpret_cast<uintptr_t>(positions) & 15u) != 0 || (reinterpret_cast<uintptr_t>(block_vids) & 15u) != 0 ||
        (reinterpret_cast<uintptr_t>(block_ranges) & 7u) != 0)
        return NXM_E_INVALID;
    if (!(cell_width > 0.f) || max_blocks == 0) return NXM_E_INVALID;
    if (n > NXM_NOALLOC_MAX_PARTICLES) return NXM_E_CAPACITY;
    *num_blocks = 0;
    unsigned char* base = nullptr;
    int rc = scratch_for_current_device(&base);
    if (rc) return rc;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        (void)cudaGetLastError();
        return NXM_E_CUDA;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    Params prm{};
    prm.dx = cell_width;
    prm.inv_dx = 1.0f / cell_width;
    prm.n = n;
    prm.block_capacity = max_blocks < kNoallocMaxBlocks ? max_blocks : kNoallocMaxBlocks;
    prm.hash_capacity = kNoallocHash;
    prm.sorted_capacity = n;

    DevPtrs P{};
    P.params = reinterpret_cast<Params*>(base + kOffParams);
    P.counters = reinterpret_cast<Counters*>(base + kOffCounters);
    P.hkey = reinterpret_cast<uint32_t*>(base + kOffHkey);
    P.hval = reinterpret_cast<uint32_t*>(base + kOffHval);
    P.bvid = reinterpret_cast<int4*>(base + kOffBvid);
    P.first = reinterpret_cast<uint32_t*>(base + kOffFirst);
    P.nprim = reinterpret_cast<uint32_t*>(base + kOffNprim);
    P.nwx = reinterpret_cast<uint32_t*>(base + kOffNwx);
    P.scan_tmp = reinterpret_cast<uint32_t*>(base + kOffScanTmp);
    P.cursors = reinterpret_cast<uint32_t*>(base + kOffCursors);
    P.nbh = reinterpret_cast<uint32_t*>(base + kOffNbh);
    P.tile_sums = reinterpret_cast<uint32_t*>(base + kOffTiles);
    P.sorted = sorted_ids;
    P.nodes = nullptr;

    LaunchCfg c{};
    c.sm_count = sms;
    c.hash_capacity = kNoallocHash;
    c.block_capacity = prm.block_capacity;
    c.particle_capacity = n;

    k_noalloc_begin<<<1, 32, 0, s>>>(prm, const_cast<Params*>(P.params), P.counters);
    if (n > 0) launch_sort_positions(P, c, reinterpret_cast<const float4*>(positions), s);
    k_noalloc_export<<<sms, 256, 0, s>>>(P.bvid, P.first, P.nprim, P.counters, reinterpret_cast<int4*>(block_vids),
                                         reinterpret_cast<uint2*>(block_ranges), max_blocks);
    Counters host{};
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(&host, P.counters, sizeof(Counters), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
        (void)cudaGetLastError();
        return NXM_E_CUDA;
    }
    // The fixed hash has two slots per block the tables hold, so a full hash
    // also means more active blocks than the tables hold: one error for both.
    if (host.status & (STATUS_HASH_FULL | STATUS_BLOCK_CAPACITY | STATUS_MISSING_BLOCK | STATUS_SORT_CAPACITY))
        return NXM_E_CAPACITY;
    *num_blocks = host.num_blocks;
    return NXM_OK;
}
