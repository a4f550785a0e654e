// Grid-wide barrier for kernels launched with cudaLaunchCooperativeKernel
// (all blocks co-resident). Arrival is an atomic counter; the last block to
// arrive bumps a generation word that the others wait on. Every wait is
// bounded: after `limit` polls (kSpinLimit unless the context sets another
// limit) the block records a timeout in *timeout and returns false, so a fault
// can never turn into a hung GPU; callers stop their work when it returns
// false and the host reports VXB_ERR_TIMEOUT.
#pragma once
#include <cstdint>

namespace vxb {

struct GridBarrier {
    unsigned int count;
    unsigned int generation;
};

constexpr unsigned int kSpinLimit = 1u << 24;  // polls of at least 32 ns: well over a second

__device__ __forceinline__ unsigned int loadVolatile(const unsigned int* p) {
    return *reinterpret_cast<const volatile unsigned int*>(p);
}

// Returns false when the wait timed out (in this block or another one).
__device__ __forceinline__ bool gridSync(GridBarrier* bar, unsigned int* timeout, unsigned int limit) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) ok = loadVolatile(timeout) == 0u;
    __syncthreads();
    if (!ok) return false;  // another block gave up: leave without waiting
    if (threadIdx.x == 0) {
        const unsigned int nblocks = gridDim.x * gridDim.y * gridDim.z;
        const unsigned int gen = loadVolatile(&bar->generation);
        __threadfence();  // release this block's writes before arriving
        if (atomicAdd(&bar->count, 1u) == nblocks - 1) {
            atomicExch(&bar->count, 0u);
            __threadfence();
            atomicAdd(&bar->generation, 1u);
        } else {
            unsigned int spins = 0;
            while (loadVolatile(&bar->generation) == gen) {
                if (++spins > limit) {
                    atomicOr(timeout, 1u);
                    ok = 0;
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();  // acquire: later loads see the other blocks' writes
    }
    __syncthreads();
    return ok != 0;
}

}  // namespace vxb
