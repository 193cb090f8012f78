// block_scan.cuh -- block-wide exclusive scans over one value per thread.
#pragma once
#include <stdint.h>

namespace csv {

// Exclusive prefix of `v` over the block in thread order; *total receives the
// block sum.  `sh` needs blockDim.x / 32 + 1 entries of shared memory.  All
// threads of the block must call it.
template <class T>
__device__ __forceinline__ T block_exclusive(T v, T* sh, T* total) {
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    T inc = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= (uint32_t)d) inc += y;
    }
    if (lane == 31) sh[w] = inc;
    __syncthreads();
    if (w == 0) {
        T s = lane < nw ? sh[lane] : T(0);
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            T y = __shfl_up_sync(0xffffffffu, s, d);
            if (lane >= (uint32_t)d) s += y;
        }
        if (lane < nw) sh[lane] = s;
    }
    __syncthreads();
    T before = (w ? sh[w - 1] : T(0)) + inc - v;
    *total = sh[nw - 1];
    __syncthreads();
    return before;
}

}  // namespace csv
