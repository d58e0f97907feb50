// scan.cuh -- block-level scan primitives (warp shuffles + shared memory).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace k3dom {

typedef unsigned __int128 u128;
typedef __int128 i128;

__device__ __forceinline__ u128 shfl_up_u128(u128 v, int delta) {
    uint64_t lo = (uint64_t)v, hi = (uint64_t)(v >> 64);
    lo = __shfl_up_sync(0xffffffffu, lo, delta);
    hi = __shfl_up_sync(0xffffffffu, hi, delta);
    return ((u128)hi << 64) | lo;
}
__device__ __forceinline__ u128 shfl_idx_u128(u128 v, int src) {
    uint64_t lo = (uint64_t)v, hi = (uint64_t)(v >> 64);
    lo = __shfl_sync(0xffffffffu, lo, src);
    hi = __shfl_sync(0xffffffffu, hi, src);
    return ((u128)hi << 64) | lo;
}

template <typename T>
__device__ __forceinline__ T shfl_up_t(T v, int d) { return __shfl_up_sync(0xffffffffu, v, d); }
template <>
__device__ __forceinline__ u128 shfl_up_t<u128>(u128 v, int d) { return shfl_up_u128(v, d); }
template <typename T>
__device__ __forceinline__ T shfl_idx_t(T v, int s) { return __shfl_sync(0xffffffffu, v, s); }
template <>
__device__ __forceinline__ u128 shfl_idx_t<u128>(u128 v, int s) { return shfl_idx_u128(v, s); }

// Inclusive warp scan (all 32 lanes active).
template <typename T>
__device__ __forceinline__ T warp_inclusive_scan(T v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        T o = shfl_up_t<T>(v, d);
        if (lane >= d) v += o;
    }
    return v;
}

// Exclusive block scan; returns the exclusive prefix of `v` and writes the block total.
// `smem` must hold NWARPS elements. All threads of the block must call it.
template <typename T, int NTHREADS>
__device__ __forceinline__ T block_exclusive_scan(T v, T* smem, T* total) {
    constexpr int NW = NTHREADS / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    T inc = warp_inclusive_scan<T>(v);
    if (lane == 31) smem[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        T s = (lane < NW) ? smem[lane] : (T)0;
        T si = warp_inclusive_scan<T>(s);
        if (lane < NW) smem[lane] = si - s;  // exclusive warp offsets
        if (lane == NW - 1) smem[NW] = si;
    }
    __syncthreads();
    T res = smem[wid] + inc - v;
    *total = smem[NW];
    __syncthreads();
    return res;
}

}  // namespace k3dom
