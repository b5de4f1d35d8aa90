// sph_noalloc.cu -- the cell-offset scan of the contact search (counts per
// cell -> exclusive offsets, the cellStart/cellEnd construction) as an entry
// point that allocates nothing.
//
// Who needs it: a caller that must not allocate device memory at the point
// of the call -- a host framework that hands out all device memory from its
// own pool and forbids driver allocations behind its back, or a steady-state
// loop in which an allocation could block on the device or fail under memory
// pressure.  The handle API allocates its scan scratch once in sph_create;
// this entry point needs no handle, so its scratch lives in a fixed
// file-scope device array instead.
//
// Scratch: one word per tile of SCAN_TILE counts plus the grand total, so at
// most MAX_TILES + 1 words (16 KiB + 4 B); counts beyond
// SPH_SCAN_STATIC_MAX are rejected.  Every call writes each scratch word
// before reading it, so nothing in the scratch has to start at zero.
// All calls on one device share the array: calls that can run at the same
// time (other streams, other host threads) race on it.
#include <cstdint>
#include <mutex>

#include <cuda_runtime.h>

#include "sphere_b200.h"

namespace {

constexpr int THREADS = 1024;
constexpr int ITEMS = 4;
constexpr uint64_t SCAN_TILE = (uint64_t)THREADS * ITEMS;                    // 4096
constexpr uint64_t MAX_TILES = SPH_SCAN_STATIC_MAX / SCAN_TILE;               // 4096
static_assert(MAX_TILES * SCAN_TILE == SPH_SCAN_STATIC_MAX, "tile count");
static_assert(MAX_TILES <= (uint64_t)THREADS * ITEMS, "one block scans the tile sums");

__device__ __align__(256) uint32_t g_tile_sums[MAX_TILES + 1];

// Exclusive scan of one value per thread over the block; *total gets the sum.
__device__ uint32_t block_scan(uint32_t v, uint32_t *smem, uint32_t *total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) smem[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const uint32_t w = lane < (int)(blockDim.x >> 5) ? smem[lane] : 0u;
        uint32_t wi = w;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, wi, o);
            if (lane >= o) wi += y;
        }
        smem[lane] = wi - w;
        if (lane == 31) smem[32] = wi;
    }
    __syncthreads();
    const uint32_t r = smem[warp] + incl - v;
    *total = smem[32];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(THREADS) k_tile_sums(const uint32_t *in, uint64_t n,
                                                       uint32_t *sums)
{
    __shared__ uint32_t smem[33];
    const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * ITEMS;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k)
        if (base + k < n) s += in[base + k];
    uint32_t total;
    block_scan(s, smem, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(THREADS) k_scan_tile_sums(uint32_t *sums, uint32_t ntiles)
{
    __shared__ uint32_t smem[33];
    uint32_t v[ITEMS], s = 0;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        const uint32_t idx = threadIdx.x * ITEMS + k;
        v[k] = idx < ntiles ? sums[idx] : 0u;
        s += v[k];
    }
    uint32_t total;
    uint32_t off = block_scan(s, smem, &total);
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        const uint32_t idx = threadIdx.x * ITEMS + k;
        if (idx < ntiles) sums[idx] = off;
        off += v[k];
    }
    if (threadIdx.x == 0) sums[ntiles] = total;
}

__global__ void __launch_bounds__(THREADS) k_tile_offsets(const uint32_t *in, uint64_t n,
                                                          const uint32_t *sums, uint32_t ntiles,
                                                          uint32_t *out)
{
    __shared__ uint32_t smem[33];
    const uint64_t base = (uint64_t)blockIdx.x * SCAN_TILE + (uint64_t)threadIdx.x * ITEMS;
    uint32_t v[ITEMS], s = 0;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        v[k] = base + k < n ? in[base + k] : 0u;
        s += v[k];
    }
    uint32_t total;
    uint32_t off = block_scan(s, smem, &total) + sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        if (base + k < n) out[base + k] = off;
        off += v[k];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = sums[ntiles];
}

// Device address of g_tile_sums, looked up with the device current and
// cached per device together with the context it belongs to: a device
// reset (cudaDeviceReset) ends the context, the module is loaded again in
// the next one and the array may move, so a call that finds another
// context current looks the address up again.  The current context is
// read through the driver's cuCtxGetCurrent, obtained from the runtime
// (no link against the driver library).
std::mutex g_lock;
constexpr int MAX_DEVICES = 64;
uint32_t *g_addr[MAX_DEVICES] = {};
void *g_ctx[MAX_DEVICES] = {};

typedef int (*CtxGetCurrentFn)(void **ctx);

void *current_context()
{
    static CtxGetCurrentFn fn = nullptr;
    static bool looked = false;
    if (!looked) {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrentFn>(f);
        looked = true;
    }
    void *ctx = nullptr;
    if (fn && fn(&ctx) != 0) ctx = nullptr;
    return ctx;
}

int scratch_address(uint32_t **out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return SPH_ERR_CUDA;
    std::lock_guard<std::mutex> guard(g_lock);
    void *ctx = current_context();
    if (!g_addr[dev] || !ctx || ctx != g_ctx[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_tile_sums) != cudaSuccess || !p) return SPH_ERR_CUDA;
        g_addr[dev] = static_cast<uint32_t *>(p);
        g_ctx[dev] = current_context();   // the lookup makes the context current if none was
    }
    *out = g_addr[dev];
    return SPH_OK;
}

}  // namespace

extern "C" int sph_cell_offsets_static(const uint32_t *counts, uint64_t n, uint32_t *offsets,
                                       void *stream)
{
    if (!offsets || (n && !counts)) return SPH_ERR_INPUT;
    if (n > SPH_SCAN_STATIC_MAX) return SPH_ERR_UNSUPPORTED;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (s) {
        // the scratch used is the current device's: the stream must be on it
        int sd = -1, cd = -1;
        if (cudaStreamGetDevice(s, &sd) != cudaSuccess || cudaGetDevice(&cd) != cudaSuccess)
            return SPH_ERR_CUDA;
        if (sd != cd) return SPH_ERR_INPUT;
    }
    uint32_t *sums = nullptr;
    const int st = scratch_address(&sums);
    if (st != SPH_OK) return st;
    const uint32_t ntiles = (uint32_t)((n + SCAN_TILE - 1) / SCAN_TILE);
    if (ntiles == 0) {
        // no counts: the single offset is 0
        return cudaMemsetAsync(offsets, 0, sizeof(uint32_t), s) == cudaSuccess ? SPH_OK
                                                                              : SPH_ERR_CUDA;
    }
    k_tile_sums<<<ntiles, THREADS, 0, s>>>(counts, n, sums);
    k_scan_tile_sums<<<1, THREADS, 0, s>>>(sums, ntiles);
    k_tile_offsets<<<ntiles, THREADS, 0, s>>>(counts, n, sums, ntiles, offsets);
    return cudaGetLastError() == cudaSuccess ? SPH_OK : SPH_ERR_CUDA;
}
