// Grid-wide barrier of the cooperative kernels (exact-order sweeps, coarse inverse), bounded: a
// block that waits longer than kBarrierSpinLimit polls, or sees the error flag already raised, raises
// it (2) and returns false, so the kernel can leave instead of hanging.  The barrier's two counters
// live in device memory that the launching code zeroes before each launch.
#pragma once

#include "common.cuh"

namespace jxcpr {

struct GridBarrier {
    unsigned int count;
    unsigned int gen;
};

static constexpr unsigned kBarrierSpinLimit = 1u << 24;

// Returns false (and raises *err) if the barrier timed out.
__device__ __forceinline__ bool grid_barrier(GridBarrier *bar, unsigned nblocks, int *err) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        volatile unsigned *vgen = &bar->gen;
        const unsigned g = *vgen;
        __threadfence();
        const unsigned prev = atomicAdd(&bar->count, 1u);
        if (prev == nblocks - 1) {
            bar->count = 0;
            __threadfence();
            atomicAdd(&bar->gen, 1u);
        } else {
            unsigned it = 0;
            while (*vgen == g) {
                if (++it > kBarrierSpinLimit || *((volatile int *)err) != 0) {
                    atomicExch(err, 2);
                    ok = 0;
                    break;
                }
                __nanosleep(20);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

}  // namespace jxcpr
