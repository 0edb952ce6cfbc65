// reduce.cuh -- deterministic warp / block / grid reductions shared by the kernels.
//
// Fixed shuffle trees inside a warp, warps summed in order inside a block, one partial per
// block in a fixed slot, and the final sum taken in slot order by the block that finishes last
// (ticket counter, reset by that block). Repeated runs with the same launch shapes give
// bit-identical results.
#pragma once

#include <cuda_runtime.h>

namespace maille {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide ordered sum of one value per thread; result valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double* sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    return t;
}

// Writes this block's partial; returns true (in every thread) in the block that finished last.
__device__ __forceinline__ bool publish_partial(double v, double* partials, unsigned int* ticket,
                                                double* sh) {
    __shared__ bool last;
    const double t = block_sum(v, sh);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = t;
        __threadfence();
        const unsigned int k = atomicAdd(ticket, 1u);
        last = (k == gridDim.x - 1);
    }
    __syncthreads();
    return last;
}

// Ordered sum of partials[0..n) by one block (every thread returns the same value).
__device__ __forceinline__ double gather_sum(const double* partials, int n, double* sh) {
    __threadfence();
    double t = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) t += __ldcg(partials + k);
    __shared__ double res;
    const double s = block_sum(t, sh);
    if (threadIdx.x == 0) res = s;
    __syncthreads();
    return res;
}

}  // namespace maille
