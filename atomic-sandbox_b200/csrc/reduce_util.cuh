// reduce_util.cuh -- deterministic in-CTA reductions (fixed shuffle tree, fixed warp order).
#pragma once
#include <cuda_runtime.h>

namespace ks {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Sum over a 1-D CTA of up to 1024 threads; the result is valid in thread 0. Contains
// __syncthreads, so every thread of the CTA must call it.
__device__ __forceinline__ double block_sum(double v) {
    __shared__ double warp_part[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    __syncthreads();  // warp_part may still be read by a previous call
    if (lane == 0) warp_part[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        s = lane < nw ? warp_part[lane] : 0.0;
        s = warp_sum(s);
    }
    return s;
}

__device__ __forceinline__ double block_max(double v) {
    __shared__ double warp_part_m[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_max(v);
    __syncthreads();
    if (lane == 0) warp_part_m[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        s = lane < nw ? warp_part_m[lane] : 0.0;
        s = warp_max(s);
    }
    return s;
}

}  // namespace ks

namespace ks {

// Maximum over a 1-D CTA for values of any sign (empty lanes count as -inf); valid in thread 0.
__device__ __forceinline__ double block_max_signed(double v) {
    __shared__ double warp_part_s[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_max(v);
    __syncthreads();
    if (lane == 0) warp_part_s[warp] = v;
    __syncthreads();
    double s = -INFINITY;
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        s = lane < nw ? warp_part_s[lane] : -INFINITY;
        s = warp_max(s);
    }
    return s;
}

}  // namespace ks
