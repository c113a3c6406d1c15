// Grid-wide barrier for kernels launched cooperatively (all CTAs co-resident), with a bounded wait.
// bar[0] counts arrivals, bar[1] is the generation; both start at zero.  A wait longer than about a
// second of clock sets *err and returns; the caller checks the result and ends the kernel.
#pragma once

namespace bemb {

__device__ __forceinline__ bool grid_barrier(unsigned* bar, int* err) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned* gen = bar + 1;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            const long long t0 = clock64();
            while (*gen == g) {
                if (clock64() - t0 > 2000000000LL) {
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
