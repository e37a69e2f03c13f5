// Block-wide sums, so that a reduction over a plane costs one atomic per
// block: thousands of warps adding into one word serialise on it.
#pragma once

#include <cuda_runtime.h>

namespace silt {

// The sum of v over the block, returned in thread 0 (others get 0). Every
// thread of the block calls it; blockDim.x is a multiple of 32, at most 1024.
template <typename V>
__device__ __forceinline__ V block_sum(V v) {
    __shared__ V part[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) part[warp] = v;
    __syncthreads();
    v = V(0);
    if (warp == 0) {
        v = lane < (int)(blockDim.x >> 5) ? part[lane] : V(0);
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    __syncthreads();  // part is reused by the next call
    return v;
}

// Adds the block's sum of v to *to (one atomic, skipped when the sum is 0).
template <typename V>
__device__ __forceinline__ void block_add(V v, V* to) {
    v = block_sum(v);
    if (threadIdx.x == 0 && v != V(0)) atomicAdd(to, v);
}

}  // namespace silt
