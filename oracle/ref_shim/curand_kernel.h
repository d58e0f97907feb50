// Test infrastructure: a stand-in for <curand_kernel.h> that serves the library's Philox draws
// to the reference's own kernels, so both run on identical random numbers.
//
// The reference draws through curand_init / curand_uniform / curand_normal
// (include/common/cuda_utils.h:27-35) from per-thread states in grid-stride loops. Here a
// state carries (thread id, call count, stage, frame, seed, draws per item); call c of thread
// tid in a launch of `stride` threads is draw k = c % dpi of item tid + (c / dpi) * stride,
// which is how the reference's grid-stride loops visit items. The harness writes the stage
// into every state before each stage it runs.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../k3dom_b200/csrc/draws.cuh"

struct curandStateShim {
    unsigned long long seed;
    unsigned int tid;
    unsigned int calls;
    unsigned int stage;
    unsigned int frame;
    unsigned int dpi;
    unsigned int pad;
};
typedef curandStateShim curandState;
typedef curandStateShim curandState_t;

__device__ inline void curand_init(unsigned long long seed, unsigned long long subsequence, unsigned long long,
                                   curandState* s) {
    s->seed = seed;
    s->tid = (unsigned int)subsequence;
    s->calls = 0;
    s->stage = 0;
    s->frame = 0;
    s->dpi = 1;
}

__device__ inline unsigned long long shim_item(curandState* s, unsigned int* k) {
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    const unsigned int dpi = s->dpi ? s->dpi : 1u;
    *k = s->calls % dpi;
    const unsigned long long item = s->tid + (unsigned long long)(s->calls / dpi) * stride;
    s->calls++;
    return item;
}

__device__ inline float curand_uniform(curandState* s) {
    unsigned int k;
    const unsigned long long item = shim_item(s, &k);
    if (s->stage == k3dom_draws::kResample) return k3dom_draws::u01(k3dom_draws::resample_word(s->seed, s->frame, item));
    return k3dom_draws::slot_uniform(s->seed, s->frame, s->stage, item, (int)k);
}

__device__ inline float curand_normal(curandState* s) {
    unsigned int k;
    const unsigned long long item = shim_item(s, &k);
    return k3dom_draws::predict_normal(s->seed, s->frame, item, (int)k);
}
