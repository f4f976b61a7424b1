// Grid-wide barrier of the persistent cooperative kernels (k_small.cu,
// k_coarse_pcg.cu): every block of the launch is resident, arrives once per
// barrier and polls a generation counter.  The wait is bounded: after `limit`
// polls (64 ns or more each) it sets bar->err and reports failure, and the
// kernel leaves its step loop instead of waiting for ever.
#pragma once

#include "tosp_internal.h"

namespace tosp {

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid-wide barrier over the co-resident blocks of a cooperative launch.
// limit: polls before the wait gives up; skip: this block does not arrive
// (a fault injected by tests: the other blocks' waits then run out).
__device__ __forceinline__ bool grid_barrier(GridBarrier *bar, unsigned nblocks, uint32_t limit, bool skip) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0 && skip) {
        s_ok = 1;
    } else if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned g = ld_acquire(&bar->gen);
        __threadfence();
        if (atomicAdd(&bar->count, 1u) == nblocks - 1) {
            atomicExch(&bar->count, 0u);
            __threadfence();
            atomicAdd(&bar->gen, 1u);
        } else {
            uint32_t it = 0;
            while (ld_acquire(&bar->gen) == g) {
                if (++it >= limit) {
                    atomicExch(&bar->err, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

}  // namespace tosp
