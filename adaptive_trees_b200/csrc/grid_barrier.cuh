// grid_barrier.cuh -- grid-wide barrier of a cooperative (co-resident) launch
// with a bounded wait.
#pragma once

#include "common.cuh"

namespace aot
{
// Barrier words (zeroed before the launch).
struct GridBarrier
{
    u32 arrived;     // CTAs at the current barrier
    u32 generation;  // barriers passed
    int error;       // a wait gave up
    int pad;
};

constexpr u32 kBarrierSpins = 1u << 22;  // polls of about 128 ns: well over 0.5 s

// Every CTA of the grid arrives; the last one opens the next generation.  A
// CTA that polls more than kBarrierSpins times (or sees another CTA's error)
// records the error and leaves; the result is false for it and for every CTA
// that reads the error after the barrier, and the kernel returns.
__device__ __forceinline__ bool gridBarrier(GridBarrier *b)
{
    __shared__ int sOk;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        volatile u32 *gen = &b->generation;
        volatile int *err = &b->error;
        const u32 g = *gen;
        __threadfence();
        if (atomicAdd(&b->arrived, 1u) == gridDim.x - 1)
        {
            atomicExch(&b->arrived, 0u);
            __threadfence();
            atomicAdd(&b->generation, 1u);
        }
        else
        {
            u32 spins = 0;
            while (*gen == g)
            {
                if (*err || ++spins > kBarrierSpins)
                {
                    atomicExch(&b->error, 1);
                    break;
                }
                __nanosleep(128);
            }
        }
        __threadfence();
        sOk = *err == 0;
    }
    __syncthreads();
    return sOk != 0;
}

template <class T>
__device__ __forceinline__ T vload(const T &x)
{
    return *static_cast<const volatile T *>(&x);
}
}  // namespace aot
