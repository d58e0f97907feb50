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
// below 2^-56 are truncated to a multiple of 2^-80. The value m * 2^(e - 150) is the 24-bit
// significand m shifted left by sh = e - 150 + kFracBits, formed in two 64-bit halves.
__device__ __forceinline__ u128 to_fixed(float f) {
    const uint32_t b = __float_as_uint(f);
    if (b >= 0x7F800000u) return 0;  // sign bit set, or Inf / NaN
    const uint32_t e = b >> 23, frac = b & 0x7FFFFFu;
    const uint64_t m = e ? (frac | 0x800000u) : frac;
    const int sh = (e ? (int)e : 1) - 150 + kFracBits;
    if (sh < 0) return (u128)(m >> min(-sh, 63));  // truncated; 0 once -sh >= 24
    if (sh > 127 - 24) return 0;                    // out of range (>= 2^47); never reached by masses
    uint64_t hi, lo;
    if (sh < 64) {
        lo = m << sh;
        hi = sh > 40 ? m >> (64 - sh) : 0ull;  // bits past position 63
    } else {
        lo = 0ull;
        hi = m << (sh - 64);
    }
    return ((u128)hi << 64) | lo;
}

// Round-to-nearest-even float of v * 2^-kFracBits. With hi != 0 the top 64 bits of v, shifted so
// that the leading one sits at bit 63, carry every bit that decides the rounding, and the bits
// shifted out below join bit 0 as a sticky bit (63 places under the rounding position); with
// hi == 0, lo converts directly. The scaling by a power of two is an add to the exponent field:
// every nonzero result lies in [2^-80, 2^48), a normal float.
__device__ __forceinline__ float from_fixed(u128 v) {
    const uint64_t hi = (uint64_t)(v >> 64), lo = (uint64_t)v;
    float f;
    int k;
    if (hi == 0ull) {
        if (lo == 0ull) return 0.0f;
        f = __ull2float_rn(lo);
        k = -kFracBits;
    } else {
        const int s = __clzll((long long)hi);
        const uint64_t top = s ? (hi << s) | (lo >> (64 - s)) : hi;
        const uint64_t rest = s ? lo << s : lo;
        f = __ull2float_rn(top | (rest != 0ull ? 1ull : 0ull));
        k = 64 - s - kFracBits;
    }
    return __int_as_float(__float_as_int(f) + k * (1 << 23));
}

}  // namespace k3dom
