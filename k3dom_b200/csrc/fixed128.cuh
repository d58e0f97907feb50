// fixed128.cuh -- conversions between non-negative floats and 128-bit fixed point with 2^-80
// resolution, the number format of the exact prefix sums (exactscan.cu, noalloc.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "scan.cuh"

namespace k3dom {

constexpr int kFracBits = 80;

// float (>= 0) -> fixed point with kFracBits fractional bits. Negative or non-finite inputs,
// and values >= 2^47, contribute 0 (they cannot occur for weights and born masses). Values
// below 2^-56 are truncated to a multiple of 2^-80.
__device__ __forceinline__ u128 to_fixed(float f) {
    uint32_t b = __float_as_uint(f);
    if (b & 0x80000000u) return 0;
    uint32_t e = b >> 23, frac = b & 0x7FFFFFu;
    if (e == 0xFFu) return 0;
    uint32_t m = e ? (frac | 0x800000u) : frac;
    int sh = (e ? (int)e : 1) - 150 + kFracBits;  // value = m * 2^(e-150)
    if (sh >= 0) {
        if (sh > 127 - 24) return 0;  // out of range (>= 2^47); never reached by masses
        return (u128)m << sh;
    }
    if (sh <= -32) return 0;
    return (u128)(m >> (-sh));
}

// Round-to-nearest-even float of v * 2^-kFracBits.
__device__ __forceinline__ float from_fixed(u128 v) {
    if (v == 0) return 0.0f;
    uint64_t hi = (uint64_t)(v >> 64), lo = (uint64_t)v;
    int lz = hi ? __clzll((long long)hi) : 64 + __clzll((long long)lo);
    u128 n = v << lz;
    uint64_t top = (uint64_t)(n >> 64);
    if ((uint64_t)n != 0) top |= 1ull;  // sticky
    float f = __ull2float_rn(top);
    return ldexpf(f, 64 - lz - kFracBits);
}

}  // namespace k3dom
