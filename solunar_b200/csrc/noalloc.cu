// noalloc.cu -- the cell sort of update_neighbors for callers that cannot allocate device memory.
//
// Some hosts give a library no way to allocate GPU memory: an engine that hands out all device
// memory from its own pool, or a plugin that only ever receives buffers from its host.  This
// entry point runs the same counting sort as slf_update_neighbors (cell keys, a count per cell,
// an exclusive scan, ranks by id within each cell) on arrays the caller owns, and keeps its
// scratch in one fixed device array declared at file scope: it never calls cudaMalloc,
// cudaFree or anything that allocates.
//
// The scratch array lives on every GPU that loads this library until the process exits.  It
// caps a call at kNoAllocMaxParticles particles whose bounding box spans at most
// kNoAllocMaxCells cells; larger calls are refused with SLF_ERR_OUT_OF_RANGE.  All calls share
// the array and it keeps what the last call left in it; the kernels clear what must start at
// zero.  Two calls whose work overlaps on the GPU (different streams, or different host threads)
// race on it.
#include <climits>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "../../include/solunar_fluid.h"
#include "fluid_device.cuh"
#include "launch.h"

namespace slf {

constexpr uint32_t kNoAllocMaxParticles = 1u << 18;  // 262,144 particles
constexpr uint32_t kNoAllocMaxCells = 1u << 20;      // 1,048,576 cells in the bounding box
constexpr uint32_t kNoAllocHeader = 64;               // bounding box, flags (u32 words)
constexpr uint32_t kNoAllocTiles = (kNoAllocMaxCells + kBlock * 8 - 1) / (kBlock * 8) + 1;

// word offsets inside the scratch array
constexpr size_t kOffLin = kNoAllocHeader;
constexpr size_t kOffSlot = kOffLin + kNoAllocMaxParticles;
constexpr size_t kOffMembers = kOffSlot + kNoAllocMaxParticles;
constexpr size_t kOffCount = kOffMembers + kNoAllocMaxParticles;
constexpr size_t kOffTiles = kOffCount + kNoAllocMaxCells + 1;
constexpr size_t kNoAllocWords = kOffTiles + kNoAllocTiles + 64;  // about 7.4 MB

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocWords];

// header words: cell box low (3), high (3), error flag
enum { kHdrLo = 0, kHdrHi = 3, kHdrError = 6 };

__global__ void k_na_reset(uint32_t* hdr) {
    if (threadIdx.x < 3) {
        reinterpret_cast<int*>(hdr)[kHdrLo + threadIdx.x] = INT_MAX;
        reinterpret_cast<int*>(hdr)[kHdrHi + threadIdx.x] = INT_MIN;
    }
    if (threadIdx.x == 0) hdr[kHdrError] = 0;
}

__device__ __forceinline__ int3 na_cell(const float* pos, uint32_t i, float radius) {
    // cell_of (src/fluid/mod.rs:526-533)
    return make_int3(__float2int_rz(floorf(pos[3 * i] / radius)), __float2int_rz(floorf(pos[3 * i + 1] / radius)),
                     __float2int_rz(floorf(pos[3 * i + 2] / radius)));
}

__global__ void k_na_bounds(const float* __restrict__ pos, uint32_t n, float radius, uint32_t* hdr) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    // whether the warp holds a particle is its own flag: a particle's cell may itself saturate
    // to INT_MAX or INT_MIN (a position of 1e30 at a small radius), so no cell value can
    // stand for "none"
    const bool any = __any_sync(0xffffffffu, i < n);
    int lo[3] = {INT_MAX, INT_MAX, INT_MAX}, hi[3] = {INT_MIN, INT_MIN, INT_MIN};
    if (i < n) {
        int3 c = na_cell(pos, i, radius);
        lo[0] = hi[0] = c.x;
        lo[1] = hi[1] = c.y;
        lo[2] = hi[2] = c.z;
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = min(lo[a], __shfl_xor_sync(0xffffffffu, lo[a], o));
            hi[a] = max(hi[a], __shfl_xor_sync(0xffffffffu, hi[a], o));
        }
    }
    if ((threadIdx.x & 31) == 0 && any) {
        int* h = reinterpret_cast<int*>(hdr);
        for (int a = 0; a < 3; ++a) {
            atomicMin(&h[kHdrLo + a], lo[a]);
            atomicMax(&h[kHdrHi + a], hi[a]);
        }
    }
}

__device__ __forceinline__ bool na_box(const uint32_t* hdr, int3& lo, int3& span) {
    const int* h = reinterpret_cast<const int*>(hdr);
    lo = make_int3(h[kHdrLo], h[kHdrLo + 1], h[kHdrLo + 2]);
    long long sx = (long long)h[kHdrHi] - lo.x + 1, sy = (long long)h[kHdrHi + 1] - lo.y + 1,
              sz = (long long)h[kHdrHi + 2] - lo.z + 1;
    if (sx <= 0 || sy <= 0 || sz <= 0) return false;
    // each side is at most 2^32 cells: bounding them first keeps the products inside 64 bits
    const long long cap = (long long)kNoAllocMaxCells;
    if (sx > cap || sy > cap || sz > cap || sx * sy > cap || sx * sy * sz > cap) return false;
    span = make_int3(int(sx), int(sy), int(sz));
    return true;
}

__global__ void k_na_count(const float* __restrict__ pos, uint32_t n, float radius, uint32_t* scratch) {
    uint32_t* hdr = scratch;
    int3 lo, span;
    if (!na_box(hdr, lo, span)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) hdr[kHdrError] = 1;
        return;
    }
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int3 c = na_cell(pos, i, radius);
    // offsets in 64 bits (a cell minus the box's low corner can pass the i32 range), and every
    // particle checked against the box before it touches the count table: a cell outside it
    // fails the call instead of writing outside the scratch array
    const long long x = (long long)c.x - lo.x, y = (long long)c.y - lo.y, z = (long long)c.z - lo.z;
    if (x < 0 || x >= span.x || y < 0 || y >= span.y || z < 0 || z >= span.z) {
        hdr[kHdrError] = 1;
        return;
    }
    uint32_t l = uint32_t((x * span.y + y) * span.z + z);
    scratch[kOffLin + i] = l;
    scratch[kOffSlot + i] = atomicAdd(&scratch[kOffCount + l], 1u);
}

__global__ void k_na_members(uint32_t n, const uint32_t* __restrict__ ids, uint32_t* scratch) {
    if (scratch[kHdrError]) return;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t l = scratch[kOffLin + i];
    scratch[kOffMembers + scratch[kOffCount + l] + scratch[kOffSlot + i]] = ids[i];
}

// order[cell start + rank of the id in its cell] = i: the (cell, id) order of mod.rs:541-550.
// A cell of k particles costs k comparisons a particle (k^2 for the cell).  Equal ids (a world's
// ids are distinct; a caller's arrays need not be) are ranked by the slot each took in its cell,
// so order is always a permutation, with repeated ids in no particular order among themselves.
__global__ void k_na_order(uint32_t n, const uint32_t* __restrict__ ids, const uint32_t* __restrict__ scratch,
                           uint32_t* __restrict__ order) {
    if (scratch[kHdrError]) return;
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t l = scratch[kOffLin + i];
    uint32_t b = scratch[kOffCount + l], e = scratch[kOffCount + l + 1];
    uint32_t id = ids[i], own = b + scratch[kOffSlot + i], rank = 0;
    for (uint32_t k = b; k < e; ++k) {
        uint32_t m = scratch[kOffMembers + k];
        rank += (m < id || (m == id && k < own)) ? 1u : 0u;
    }
    order[b + rank] = i;
}

namespace {

std::mutex g_noalloc_mutex;
uint32_t* g_noalloc_ptr[256] = {};  // device address of the scratch array, per device ordinal
thread_local uint32_t h_noalloc_error;

int32_t na_fail(int32_t code, const char* what, cudaError_t e = cudaSuccess) {
    std::string msg = what;
    if (e != cudaSuccess) msg += std::string(": ") + cudaGetErrorString(e);
    set_last_error(msg);
    return code;
}

// The scratch array's device address on the current device, looked up once per device.
int32_t scratch_on_current_device(uint32_t** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return na_fail(SLF_ERR_CUDA, "cudaGetDevice", e);
    if (dev < 0 || dev >= 256) return na_fail(SLF_ERR_CUDA, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return na_fail(SLF_ERR_CUDA, "cudaGetSymbolAddress", e);
        g_noalloc_ptr[dev] = static_cast<uint32_t*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return SLF_OK;
}

}  // namespace

}  // namespace slf

extern "C" int32_t slf_sort_by_cell_noalloc(const float* positions, const uint32_t* ids, uint64_t n, float radius,
                                            uint32_t* order, void* stream) {
    using namespace slf;
    if (n == 0) return SLF_OK;
    if (!positions || !ids || !order) return na_fail(SLF_ERR_INVALID_ARGUMENT, "null device pointer");
    if (!(radius > 0.0f) || !std::isfinite(radius)) return na_fail(SLF_ERR_INVALID_ARGUMENT, "radius must be positive");
    if (n > kNoAllocMaxParticles) return na_fail(SLF_ERR_OUT_OF_RANGE, "more particles than the scratch holds");
    uint32_t* scratch = nullptr;
    int32_t st = scratch_on_current_device(&scratch);
    if (st != SLF_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    uint32_t m = uint32_t(n);
    uint32_t blocks = (m + kBlock - 1) / kBlock;
    k_na_reset<<<1, 32, 0, s>>>(scratch);
    cudaError_t e = cudaMemsetAsync(scratch + kOffCount, 0, (size_t(kNoAllocMaxCells) + 1) * 4, s);
    if (e != cudaSuccess) return na_fail(SLF_ERR_CUDA, "clearing the cell counts", e);
    k_na_bounds<<<blocks, kBlock, 0, s>>>(positions, m, radius, scratch);
    k_na_count<<<blocks, kBlock, 0, s>>>(positions, m, radius, scratch);
    launch_exclusive_scan(scratch + kOffCount, kNoAllocMaxCells, scratch + kOffTiles, s);
    k_na_members<<<blocks, kBlock, 0, s>>>(m, ids, scratch);
    k_na_order<<<blocks, kBlock, 0, s>>>(m, ids, scratch, order);
    e = cudaGetLastError();
    if (e != cudaSuccess) return na_fail(SLF_ERR_CUDA, "launching the cell sort", e);
    e = cudaMemcpyAsync(&h_noalloc_error, scratch + kHdrError, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return na_fail(SLF_ERR_CUDA, "finishing the cell sort", e);
    if (h_noalloc_error) return na_fail(SLF_ERR_OUT_OF_RANGE, "particles spread over more cells than the scratch holds");
    return SLF_OK;
}
