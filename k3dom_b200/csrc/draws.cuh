// draws.cuh -- counter-based random draws of the K3DOM update.
//
// The reference draws from per-thread cuRAND XORWOW states (include/common/cuda_utils.h:27-35,
// seeded at src/common/dom.cu:96), so its numbers depend on the launch shape. Here every
// draw is a pure function of (seed, frame, stage, item, k) through Philox4x32-10
// (J. K. Salmon, M. A. Moraes, R. O. Dror, D. E. Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11), so any kernel layout produces the same stream and a CPU oracle can
// recompute the uniforms exactly.
//
//  * uniform: u = ((r >> 8) + 1) * 2^-24 in (0, 1], the half-open convention of
//    curand_uniform that cuda_utils.h:27-31 relies on; exact in FP32.
//  * normal: Box-Muller (G. E. P. Box, M. E. Muller, 1958) on two uniforms,
//    rho = sqrt(-2 ln u1), z0 = rho cos(2 pi u2), z1 = rho sin(2 pi u2).
//
// Stage map (item = particle / slot / draw index):
//  1 prediction : 6 normals per particle (predict.cu:20-25 order: pos x,y,z, vel x,y,z).
//                 normal k uses block k/4 and the uniform pair (k%4)/2; even k -> cos, odd -> sin.
//  2 first-frame velocities : 3 uniforms per slot (init_new_particles.cu:77-79), block 0, r[k].
//  3 birth velocities : 3 uniforms per slot (init_new_particles.cu:147-149), block 0, r[k].
//  4 resampling : 1 uniform per draw i (resampling.cu:48-51); r[i % 4] of block 0 of item i/4.
// This header is shared with the draw-injection shim used to run the reference's own CUDA
// on identical draws.
#pragma once
#include <stdint.h>

#ifndef K3DOM_HD
#define K3DOM_HD __host__ __device__ __forceinline__
#endif

namespace k3dom_draws {

enum Stage : uint32_t { kPredict = 1, kInitVel = 2, kBirthVel = 3, kResample = 4 };

struct U4 { uint32_t x, y, z, w; };

K3DOM_HD uint32_t mulhilo(uint32_t a, uint32_t b, uint32_t* hi) {
#ifdef __CUDA_ARCH__
    *hi = __umulhi(a, b);
    return a * b;
#else
    uint64_t p = (uint64_t)a * (uint64_t)b;
    *hi = (uint32_t)(p >> 32);
    return (uint32_t)p;
#endif
}

// Philox4x32 with 10 rounds.
K3DOM_HD U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, hi1;
        uint32_t lo0 = mulhilo(M0, c.x, &hi0);
        uint32_t lo1 = mulhilo(M1, c.z, &hi1);
        U4 n;
        n.x = hi1 ^ c.y ^ k0;
        n.y = lo1;
        n.z = hi0 ^ c.w ^ k1;
        n.w = lo0;
        c = n;
        k0 += W0;
        k1 += W1;
    }
    return c;
}

K3DOM_HD U4 block(uint64_t seed, uint32_t frame, uint32_t stage, uint64_t item, uint32_t blk) {
    U4 c;
    c.x = (uint32_t)item;
    c.y = (uint32_t)(item >> 32);
    c.z = blk | (stage << 24);
    c.w = frame;
    return philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
}

// (0, 1] with 24 significant bits; exact in float.
K3DOM_HD float u01(uint32_t r) { return (float)((r >> 8) + 1u) * 5.9604644775390625e-08f; }

// 1 - u01(r) as an integer on the 2^-24 grid, in [0, 2^24): the sort key of a resampling draw.
K3DOM_HD uint32_t one_minus_u01_key(uint32_t r) { return 0xFFFFFFu - (r >> 8); }

K3DOM_HD uint32_t pick(const U4& v, int i) {
    return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}

// Uniform k (0..3) of the single-block stages 2 and 3.
K3DOM_HD float slot_uniform(uint64_t seed, uint32_t frame, uint32_t stage, uint64_t item, int k) {
    return u01(pick(block(seed, frame, stage, item, 0), k));
}

// Resampling draw i as the raw 32-bit Philox word.
K3DOM_HD uint32_t resample_word(uint64_t seed, uint32_t frame, uint64_t i) {
    return pick(block(seed, frame, kResample, i >> 2, 0), (int)(i & 3));
}

#ifdef __CUDACC__
// Box-Muller pair from two words; rounding pinned with _rn intrinsics so that every
// build of this header yields identical bits.
__device__ __forceinline__ void box_muller(uint32_t ra, uint32_t rb, float* z0, float* z1) {
    float u1 = u01(ra);
    float u2 = u01(rb);
    float rho = sqrtf(__fmul_rn(-2.0f, logf(u1)));
    float s, c;
    sincospif(__fmul_rn(2.0f, u2), &s, &c);
    *z0 = __fmul_rn(rho, c);
    *z1 = __fmul_rn(rho, s);
}

// All six prediction normals of one particle, in the order pos x,y,z, vel x,y,z.
__device__ __forceinline__ void predict_normals(uint64_t seed, uint32_t frame, uint64_t item,
                                                float n[6]) {
    U4 b0 = block(seed, frame, kPredict, item, 0);
    U4 b1 = block(seed, frame, kPredict, item, 1);
    box_muller(b0.x, b0.y, &n[0], &n[1]);
    box_muller(b0.z, b0.w, &n[2], &n[3]);
    box_muller(b1.x, b1.y, &n[4], &n[5]);
}

// Normal k (0..5) alone; used by the draw-injection shim, equal to predict_normals()[k].
__device__ __forceinline__ float predict_normal(uint64_t seed, uint32_t frame, uint64_t item, int k) {
    U4 b = block(seed, frame, kPredict, item, (uint32_t)(k >> 2));
    int p = (k & 3) >> 1;
    float z0, z1;
    box_muller(pick(b, 2 * p), pick(b, 2 * p + 1), &z0, &z1);
    return (k & 1) ? z1 : z0;
}
#endif

}  // namespace k3dom_draws
