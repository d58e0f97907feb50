// exactscan.cu -- inclusive prefix sums of non-negative floats that are exact and
// order-independent.
//
// The reference forms these sums with thrust::inclusive_scan in FP32
// (include/common/common.h:7-18, called at src/common/dom.cu:215-217 for born masses and
// :268-273 for the joint weights). Their rounding depends on CUB's tiling, and the integer
// results derived from them (birth slot boundaries, init_new_particles.cu:14-27; ancestor
// indices, resampling.cu:55-68) inherit that dependence. Here every element is converted
// exactly to a 128-bit fixed-point integer with 2^-80 resolution, the integers are summed
// (associative), and each prefix is rounded once to the nearest float. The result is the
// correctly rounded exact prefix, independent of the launch shape, so a CPU oracle
// reproduces it bit for bit.
#include <cuda_runtime.h>

#include "common.cuh"
#include "fixed128.cuh"
#include "internal.h"
#include "scan.cuh"

#include <algorithm>
#include <cstdint>
#include <vector>

namespace k3dom {

constexpr int kExThreads = 256;
constexpr int kExItems = 8;
constexpr int kExTile = kExThreads * kExItems;
struct TwoSeg {
    const float* a;
    long na;
    const float* b;
    __device__ __forceinline__ float operator()(long i) const { return i < na ? a[i] : b[i - na]; }
};

__global__ void exact_tile_sums(TwoSeg in, long n, u128* __restrict__ tile_sums) {
    __shared__ u128 sm[kExThreads / 32 + 1];
    const long base = (long)blockIdx.x * kExTile;
    u128 s = 0;
#pragma unroll
    for (int j = 0; j < kExItems; ++j) {
        long i = base + (long)j * kExThreads + threadIdx.x;
        if (i < n) s += to_fixed(in(i));
    }
    u128 tot;
    block_exclusive_scan<u128, kExThreads>(s, sm, &tot);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

__global__ void exact_tile_offsets(u128* __restrict__ tile_sums, int ntiles) {
    __shared__ u128 sm[kExThreads / 32 + 1];
    u128 carry = 0;
    for (int b = 0; b < ntiles; b += kExThreads) {
        int i = b + threadIdx.x;
        u128 v = (i < ntiles) ? tile_sums[i] : (u128)0;
        u128 tot;
        u128 ex = block_exclusive_scan<u128, kExThreads>(v, sm, &tot);
        if (i < ntiles) tile_sums[i] = carry + ex;
        carry += tot;
    }
}

__global__ void exact_apply(TwoSeg in, long n, const u128* __restrict__ tile_off,
                            float* __restrict__ out) {
    __shared__ u128 sm[kExThreads / 32 + 1];
    const long base = (long)blockIdx.x * kExTile + (long)threadIdx.x * kExItems;
    u128 v[kExItems];
    u128 s = 0;
#pragma unroll
    for (int j = 0; j < kExItems; ++j) {
        long i = base + j;
        v[j] = (i < n) ? to_fixed(in(i)) : (u128)0;
        s += v[j];
    }
    u128 tot;
    u128 run = tile_off[blockIdx.x] + block_exclusive_scan<u128, kExThreads>(s, sm, &tot);
#pragma unroll
    for (int j = 0; j < kExItems; ++j) {
        long i = base + j;
        run += v[j];
        if (i < n) out[i] = from_fixed(run);
    }
}

// ---------------------------------------------------------------- segmented, table driven
// A scan plan lists tiles of at most kExTile elements; each tile reads one contiguous input
// range and writes one contiguous output range, and names the first tile of its segment.
// Output = exact prefix within the segment, rounded once: the global prefix in 128-bit fixed
// point minus the global prefix at the segment's first tile, both exact.
constexpr int kExGroup = kExThreads * kExItems;  // tiles per group of the offset pass

__global__ void exact_tab_sums(const ExactTile* __restrict__ tiles, int nt, u128* __restrict__ tsum) {
    __shared__ u128 sm[kExThreads / 32 + 1];
    const int b = blockIdx.x;
    if (b >= nt) return;
    const ExactTile t = tiles[b];
    u128 s = 0;
#pragma unroll
    for (int j = 0; j < kExItems; ++j) {
        const int i = j * kExThreads + threadIdx.x;
        if (i < t.n) s += to_fixed(t.in[i]);
    }
    u128 tot;
    block_exclusive_scan<u128, kExThreads>(s, sm, &tot);
    if (threadIdx.x == 0) tsum[b] = tot;
}

// Within each group of kExGroup tiles: tile sums -> exclusive prefixes; group totals out.
__global__ void exact_tab_groups(u128* __restrict__ tsum, int nt, u128* __restrict__ gsum) {
    __shared__ u128 sm[kExThreads / 32 + 1];
    const int base = blockIdx.x * kExGroup + threadIdx.x * kExItems;
    u128 v[kExItems];
    u128 s = 0;
#pragma unroll
    for (int j = 0; j < kExItems; ++j) {
        v[j] = (base + j < nt) ? tsum[base + j] : (u128)0;
        s += v[j];
    }
    u128 tot;
    u128 run = block_exclusive_scan<u128, kExThreads>(s, sm, &tot);
#pragma unroll
    for (int j = 0; j < kExItems; ++j) {
        if (base + j < nt) tsum[base + j] = run;
        run += v[j];
    }
    if (threadIdx.x == 0) gsum[blockIdx.x] = tot;
}

__device__ __forceinline__ u128 group_prefix(const u128* __restrict__ gsum, int g) {
    // sum of gsum[0..g): warp 0 reduces, result broadcast through shared memory
    __shared__ u128 s_r;
    if (threadIdx.x < 32) {
        u128 a = 0;
        for (int i = threadIdx.x; i < g; i += 32) a += gsum[i];
        a = warp_inclusive_scan<u128>(a);
        if (threadIdx.x == 31) s_r = a;
    }
    __syncthreads();
    const u128 r = s_r;
    __syncthreads();
    return r;
}

// 4 CTAs per SM (64 registers): the pass waits on its loads with few warps otherwise. CLEAR: the
// tile's sign-bit inputs (which the scan counts as 0) are set to +0 in place.
template <bool CLEAR>
__global__ void __launch_bounds__(kExThreads, 4) exact_tab_apply(const ExactTile* __restrict__ tiles, int nt,
                                                                const u128* __restrict__ tsum,
                                const u128* __restrict__ gsum) {
    __shared__ u128 sm[kExThreads / 32 + 1];
    const int b = blockIdx.x;
    const ExactTile t = tiles[b];
    const u128 pre_b = group_prefix(gsum, b / kExGroup) + tsum[b];
    const int f = t.seg_first;
    const u128 pre_f = group_prefix(gsum, f / kExGroup) + tsum[f];
    const int base = threadIdx.x * kExItems;
    // the inputs stay in registers as floats and are converted twice (cheaper than holding
    // eight 128-bit values across the block scan)
    // a full tile with 16-byte aligned ranges moves its 8 values per thread as two float4
    const bool vec = t.n == kExTile &&
                     ((reinterpret_cast<uintptr_t>(t.in) | reinterpret_cast<uintptr_t>(t.out)) & 15u) == 0;
    float x[kExItems];
    if (vec) {
        const float4* p = reinterpret_cast<const float4*>(t.in + base);
        const float4 a = p[0], c = p[1];
        x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w;
        x[4] = c.x; x[5] = c.y; x[6] = c.z; x[7] = c.w;
    } else {
#pragma unroll
        for (int j = 0; j < kExItems; ++j) x[j] = (base + j < t.n) ? t.in[base + j] : 0.0f;
    }
    if (CLEAR) {
#pragma unroll
        for (int j = 0; j < kExItems; ++j)
            if (signbit(x[j]) && base + j < t.n) t.in[base + j] = 0.0f;
    }
    u128 s = 0;
#pragma unroll
    for (int j = 0; j < kExItems; ++j) s += to_fixed(x[j]);
    u128 tot;
    u128 run = (pre_b - pre_f) + block_exclusive_scan<u128, kExThreads>(s, sm, &tot);
    float y[kExItems];
#pragma unroll
    for (int j = 0; j < kExItems; ++j) {
        run += to_fixed(x[j]);
        y[j] = from_fixed(run);
    }
    if (vec) {
        float4* q = reinterpret_cast<float4*>(t.out + base);
        q[0] = make_float4(y[0], y[1], y[2], y[3]);
        q[1] = make_float4(y[4], y[5], y[6], y[7]);
    } else {
#pragma unroll
        for (int j = 0; j < kExItems; ++j)
            if (base + j < t.n) t.out[base + j] = y[j];
    }
}

int exact_plan_tiles(long n) { return div_up(n, kExTile); }

void exact_plan_add(std::vector<ExactTile>& plan, float* const* in, const long* n, int pieces, float* out) {
    const int first = (int)plan.size();
    long o = 0;
    for (int k = 0; k < pieces; ++k) {
        for (long i = 0; i < n[k]; i += kExTile) {
            ExactTile t;
            t.in = in[k] + i;
            t.out = out + o + i;
            t.n = (int)std::min<long>(kExTile, n[k] - i);
            t.seg_first = first;
            plan.push_back(t);
        }
        o += n[k];
    }
}

size_t exact_plan_scratch_bytes(int ntiles) {
    return ((size_t)ntiles + (size_t)div_up(ntiles, kExGroup) + 2) * sizeof(u128);
}

cudaError_t exact_scan_plan(const ExactTile* tiles, int nt, void* scratch, cudaStream_t st, bool clear_signed) {
    if (nt <= 0) return cudaSuccess;
    u128* tsum = reinterpret_cast<u128*>(scratch);
    u128* gsum = tsum + nt;
    const int ng = div_up(nt, kExGroup);
    ++g_launches;
    exact_tab_sums<<<nt, kExThreads, 0, st>>>(tiles, nt, tsum);
    ++g_launches;
    exact_tab_groups<<<ng, kExThreads, 0, st>>>(tsum, nt, gsum);
    ++g_launches;
    if (clear_signed)
        exact_tab_apply<true><<<nt, kExThreads, 0, st>>>(tiles, nt, tsum, gsum);
    else
        exact_tab_apply<false><<<nt, kExThreads, 0, st>>>(tiles, nt, tsum, gsum);
    return cudaGetLastError();
}

int exact_scan_tiles(long n) { return div_up(n, kExTile); }
size_t exact_scan_scratch_bytes(long n) { return (size_t)(exact_scan_tiles(n) + 1) * sizeof(u128); }

static cudaError_t exact_scan_impl(TwoSeg in, long n, float* out, void* scratch, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    int nt = exact_scan_tiles(n);
    u128* ts = reinterpret_cast<u128*>(scratch);
    ++g_launches;
    exact_tile_sums<<<nt, kExThreads, 0, st>>>(in, n, ts);
    ++g_launches;
    exact_tile_offsets<<<1, kExThreads, 0, st>>>(ts, nt);
    ++g_launches;
    exact_apply<<<nt, kExThreads, 0, st>>>(in, n, ts, out);
    return cudaGetLastError();
}

cudaError_t exact_scan_float(const float* in, float* out, long n, void* scratch, cudaStream_t st) {
    TwoSeg s{in, n, in};
    return exact_scan_impl(s, n, out, scratch, st);
}

cudaError_t exact_scan_float2(const float* a, long na, const float* b, long nb, float* out,
                              void* scratch, cudaStream_t st) {
    TwoSeg s{a, na, b};
    return exact_scan_impl(s, na + nb, out, scratch, st);
}

}  // namespace k3dom
