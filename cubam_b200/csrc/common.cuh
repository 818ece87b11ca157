// Shared definitions of the B200 BAM reader kernels (sm_100a).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/cubam_b200.h"

// The current value of a launch parameter (abi.cu; cb_set_param / cb_get_param).
int64_t cb_param(int key);

namespace cb {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ uint32_t ld_u16(const uint8_t* b, long long o) {
    return (uint32_t)b[o] | ((uint32_t)b[o + 1] << 8);
}
__device__ __forceinline__ uint32_t ld_u32(const uint8_t* b, long long o) {
    return (uint32_t)b[o] | ((uint32_t)b[o + 1] << 8) | ((uint32_t)b[o + 2] << 16) | ((uint32_t)b[o + 3] << 24);
}

// Exclusive prefix sum over the 32 lanes of a warp.
template <class T> __device__ __forceinline__ T warp_exclusive_scan(T v, T& total) {
    const int lane = threadIdx.x & 31;
    T x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        T y = __shfl_up_sync(FULL, x, d);
        if (lane >= d) x += y;
    }
    total = __shfl_sync(FULL, x, 31);
    return x - v;
}

// Exclusive prefix sum over a block of NT threads (NT a multiple of 32, at most 1024).
template <int NT, class T> __device__ __forceinline__ T block_exclusive_scan(T v, T& total, T* smem32) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    T wt;
    T x = warp_exclusive_scan(v, wt);
    if (lane == 0) smem32[warp] = wt;
    __syncthreads();
    if (warp == 0) {
        T s = lane < NT / 32 ? smem32[lane] : T(0);
        T t;
        T e = warp_exclusive_scan(s, t);
        if (lane < NT / 32) smem32[lane] = e;
        if (lane == 0) smem32[32] = t;
    }
    __syncthreads();
    x += smem32[warp];
    total = smem32[32];
    __syncthreads();
    return x;
}

}  // namespace cb
