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

// Bytes of device data read straight from global memory (the accessor form of ld_u16 / ld_u32).
struct GlobalBytes {
    const uint8_t* g;
    __device__ __forceinline__ uint32_t u8(long long o) const { return g[o]; }
    __device__ __forceinline__ uint32_t u16(long long o) const { return ld_u16(g, o); }
    __device__ __forceinline__ uint32_t u32(long long o) const { return ld_u32(g, o); }
};

// Bytes of device data from a copy staged in shared memory where it covers them, else from global
// memory.  s[0] holds data byte r0 and data + r0 is 16-byte aligned, so byte o sits in word
// (o - r0) / 4 of the copy; [r0, hi) is staged, and the copy has at least 4 bytes after hi - r0
// rounded up to 4 (word reads fetch the word after the one holding o).
struct StagedBytes {
    const uint8_t* g;
    const uint8_t* s;
    long long r0, hi;
    __device__ __forceinline__ bool in(long long o, int sz) const { return o >= r0 && o + sz <= hi; }
    __device__ __forceinline__ uint32_t u8(long long o) const { return in(o, 1) ? s[o - r0] : __ldg(g + o); }
    __device__ __forceinline__ uint32_t u16(long long o) const {
        return in(o, 2) ? (uint32_t)s[o - r0] | ((uint32_t)s[o - r0 + 1] << 8) : ld_u16(g, o);
    }
    __device__ __forceinline__ uint32_t u32(long long o) const {
        if (in(o, 4)) {
            const long long r = o - r0;
            const uint32_t* w = reinterpret_cast<const uint32_t*>(s + (r & ~3LL));
            return __funnelshift_r(w[0], w[1], (unsigned)(r & 3) * 8);
        }
        return ld_u32(g, o);
    }
};

// The same staged window addressed by 32-bit offsets x from its start r0 (x >= 0): s holds bytes
// [0, wlen), g = data + r0 reaches the rest.  For walks that stay within 2^30 bytes of r0.
struct WindowBytes {
    const uint8_t* g;
    const uint8_t* s;
    int wlen;
    __device__ __forceinline__ uint32_t u8(int x) const { return x < wlen ? s[x] : __ldg(g + x); }
    __device__ __forceinline__ uint32_t u16(int x) const {
        return x + 2 <= wlen ? (uint32_t)s[x] | ((uint32_t)s[x + 1] << 8) : ld_u16(g, x);
    }
    __device__ __forceinline__ uint32_t u32(int x) const {
        if (x + 4 <= wlen) {
            const uint32_t* w = reinterpret_cast<const uint32_t*>(s + (x & ~3));
            return __funnelshift_r(w[0], w[1], (unsigned)(x & 3) * 8);
        }
        return ld_u32(g, x);
    }
};

// Copy the data bytes [lo, hi) to shared memory `st` with the warp's asynchronous 16-byte copies
// (cp.async: coalesced, all in flight at once, no registers held; the first and last 16-byte blocks
// are copied whole, which never leaves the pages holding the range), then wait for them and sync the
// warp; returns the window start r0 (lo rounded down to a 16-byte address).
__device__ __forceinline__ long long stage_bytes(const uint8_t* b, long long lo, long long hi, uint4* st) {
    const int lane = threadIdx.x & 31;
    const long long r0 = lo - (long long)(reinterpret_cast<uintptr_t>(b + lo) & 15);
    const long long nblk = hi > lo ? (hi - r0 + 15) >> 4 : 0;
    const uint4* src = reinterpret_cast<const uint4*>(b + r0);
    for (long long j = lane; j < nblk; j += 32) {
        const unsigned dst = (unsigned)__cvta_generic_to_shared(st + j);
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src + j) : "memory");
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncwarp();
    return r0;
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
