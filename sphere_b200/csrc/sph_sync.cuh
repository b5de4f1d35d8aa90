// sph_sync.cuh -- a grid-wide barrier among the blocks of one cooperative
// launch, for the persistent kernels (the list step, the Darcy solve).
#pragma once

#include <cstdint>

#include "sph_device.cuh"
#include "sph_internal.h"

namespace sph {

__device__ __forceinline__ unsigned long long now_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// A grid-wide barrier with a time limit: the blocks of one launch (all
// resident: the launch is cooperative) count in, the last one opens the
// next generation; a block that waits longer than G.limit_ns raises
// SPH_ERR_TIMEOUT and returns false (its kernel then ends, and so do the
// others, at this barrier or the next), so a block that never arrives does
// not hang the device.
__device__ __forceinline__ bool grid_barrier(const GridSync &G, uint32_t nblocks, uint32_t *err)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        volatile uint32_t *gen = G.gen;
        const uint32_t g = *gen;
        __threadfence();
        if (atomicAdd(G.count, 1u) == nblocks - 1u) {
            atomicExch(G.count, 0u);
            __threadfence();
            atomicAdd(G.gen, 1u);
        } else {
            const unsigned long long t0 = now_ns();
            while (*gen == g) {
                if (now_ns() - t0 > G.limit_ns) {
                    ok = 0;
                    raise_flag(err, SPH_ERR_TIMEOUT);
                    break;
                }
                __nanosleep(128);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ unsigned long long ld_acquire_gpu_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// A grid-wide barrier on an arrival counter that only grows (zeroed before
// the launch): at its n-th barrier (n = 1, 2, ...) each block adds one with
// a release reduction, which needs no answer, and polls the counter with
// acquire loads until it reaches n x nblocks.  Against the generation
// barrier above this saves the load of the generation before the arrival
// and the last block's publication after it.  `arrive` runs on thread 0
// between the block barrier and the arrival, so what it writes (and what
// the block wrote before the barrier) is released with the arrival.  Same
// time limit and error as above.
template <class F>
__device__ __forceinline__ bool grid_sync_count(unsigned long long *ctr, unsigned long long target,
                                                unsigned long long limit_ns, uint32_t *err, F arrive)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        arrive();
        asm volatile("red.release.gpu.global.add.u64 [%0], 1;" ::"l"(ctr) : "memory");
        const unsigned long long t0 = now_ns();
        uint32_t polls = 0;
        while (ld_acquire_gpu_u64(ctr) < target) {
            if ((++polls & 63u) == 0u && now_ns() - t0 > limit_ns) {
                ok = 0;
                raise_flag(err, SPH_ERR_TIMEOUT);
                break;
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

}  // namespace sph
