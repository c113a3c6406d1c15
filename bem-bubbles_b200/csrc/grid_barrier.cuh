// Grid-wide barrier for kernels launched cooperatively (all CTAs co-resident), with a bounded wait.
// bar[0] counts arrivals, bar[1] is the generation; both start at zero.  A wait longer than `limit`
// SM clock cycles (GRID_WAIT_CYCLES, about a second, unless the context sets another bound) sets
// *err and returns false; the caller then ends the kernel.  Every CTA still arrives at the barrier
// it reached, so the last arrival resets the count and bumps the generation as usual.  A CTA that
// passed that barrier before the error word was set leaves at the next one, where the CTA that gave
// up never arrives, by its own bounded wait: an expired wait ends the kernel within two limits, with
// no CTA left waiting.
#pragma once

namespace bemb {

constexpr long long GRID_WAIT_CYCLES = 2000000000LL;

// genw: the generation word; callers whose CTAs are many keep it on another cache line than the
// arrival count (bar[0]), so that the polling does not queue behind the arrivals' atomics, and poll
// with a short sleep (sleep_ns > 0).
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned* genw, int* err, long long limit,
                                             unsigned sleep_ns = 0) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = genw;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(genw, 1u);
        } else {
            const long long t0 = clock64();
            while (*gen == g) {
                if (sleep_ns) __nanosleep(sleep_ns);
                if (clock64() - t0 > limit) {
                    atomicExch(err, 1);
                    break;
                }
            }
        }
        __threadfence();
        s_ok = *(volatile int*)err == 0;
    }
    __syncthreads();
    return s_ok != 0;
}

}  // namespace bemb
