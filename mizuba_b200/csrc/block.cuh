// Block-wide primitives for 1024-thread (or smaller, multiple-of-32) blocks.
#pragma once

#include <cstdint>

namespace mzb
{

__device__ __forceinline__ unsigned lanemask_lt()
{
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Exclusive prefix sum of v over the block; *total receives the block sum.
// smem must hold 33 uint32.  Contains __syncthreads().
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *smem, uint32_t *total)
{
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned nwarps = (blockDim.x + 31) >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= unsigned(o)) x += y;
    }
    if (lane == 31) smem[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = (lane < nwarps) ? smem[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= unsigned(o)) w += y;
        }
        if (lane < nwarps) smem[lane] = w; // inclusive warp totals
        if (lane == 31) smem[32] = w;
    }
    __syncthreads();
    const uint32_t before = (warp == 0) ? 0 : smem[warp - 1];
    *total = smem[32];
    const uint32_t r = before + x - v;
    __syncthreads();
    return r;
}

} // namespace mzb
