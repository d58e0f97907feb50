// evidence.cu -- measurement evidence and the per-cell mass update, for every scene of a batch
// in one launch per kernel.
//
// K3DOM: Bayesian kernel inference (BGKI, src/k3dom/kernel/mass_update.cu:32-77) followed by
// predict_mass / update_mass / separate_newborn_part (:79-150), with the per-cell parts of
// updatePersistentParticlesKernel2 (update_persistent_particles.cu:28-44) and
// statisticalMomentsKernel2 (statistical_moments.cu:36-63) fused into the same pass.
// DS-PHD/MIB: calcMeasurementGridKernel (src/dsphdmib/kernel/measurement_grid.cu:64-162)
// followed by gridCellPredictionUpdateKernel (src/dsphdmib/kernel/mass_update.cu:46-87).
//
// The reference evaluates every (cell, point) pair: C x N (2.5e11 at 2.1M cells / 120k
// points). Both evidence models have compact support -- the sparse kernel is zero beyond
// ls, the DS window is 0.866 res wide -- so each ray is binned to the tiles of cells its
// support can reach (segment sensor->point with radius ls for K3DOM, the half-line through
// the point with the window radius for DS). Tiles of all scenes share one global numbering
// (scene tile offset + local tile), so one pass builds every scene's lists. K3DOM places each
// ray into its tiles' ranges through per-block tallies of each tile (its exact sums make the order
// within a tile immaterial); DS keeps a tile's rays in input order (a stable sort by tile), as
// its first-100 rule needs. One CTA takes one (tile, chunk of rays) work item
// from a device work counter and stages the chunk's rays in shared memory; its warps pull the
// tile's 4x4x2-cell sub-blocks from a block-local counter, cull 32 rays at a time with one
// ballot, and every lane evaluates the surviving rays for its own cell.
//
// K3DOM evidence is summed in fixed point: each kernel value is rounded once to an integer
// number of units of 2^-k sigma (the table carries the scale), summed exactly in 64-bit
// integers (per lane, then atomics across sub-blocks and chunks), so a cell's evidence is the
// same for any tiling, chunking, ray order or scheduling. The
// last CTA to finish a tile's chunks runs the cell update for the whole tile. No block ever
// waits on another.
#include <cuda_runtime.h>
#include <math.h>

#include <algorithm>
#include <cmath>
#include <cstddef>

#include "common.cuh"
#include "internal.h"
#include "scan.cuh"

namespace k3dom {

constexpr int kChunk = 1024;      // largest number of rays per work item
constexpr int kKernelTab = 512;  // intervals of the sparse-kernel table over u = d^2 / ls^2
constexpr int kKernelTabEntries = kKernelTab + 1;  // + a zero entry at u = 1
static_assert(kKernelTabEntries == kKernelTableSize, "kernel table size");
constexpr int kEvThreads = 256;
constexpr int kEvWarps = kEvThreads / 32;
constexpr int kSmallChunk = 256;  // items up to this many rays run in CTAs of kSmallWarps warps
constexpr int kSmallWarps = 4;
constexpr int kDsMaxNeighbors = 100;  // measurement_grid.cu:87

// ================================================================ binning
struct BinGeom {
    float ax, ay, az;  // sensor in cell-index space (cell centre ix sits at u = ix)
    float R;           // support radius in cells
    int G, Gz, tx, ty, tz, ntx, nty, ntz;
};

// Whether the segment a + t d, t in [t0, t1], meets the box [l, h]; inv[k] = 1 / d[k] (unused
// where d[k] = 0).
__device__ __forceinline__ bool seg_box(const float a[3], const float d[3], const float inv[3], const float l[3],
                                        const float h[3], float t0, float t1) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (d[k] == 0.0f) {
            if (a[k] < l[k] || a[k] > h[k]) return false;
        } else {
            const float e0 = (l[k] - a[k]) * inv[k], e1 = (h[k] - a[k]) * inv[k];
            t0 = fmaxf(t0, fminf(e0, e1));
            t1 = fminf(t1, fmaxf(e0, e1));
        }
    }
    return t0 <= t1;
}

// v[k] for k in {0, 1, 2} by selects (a run-time index into a local array would go through
// local memory).
template <typename T>
__device__ __forceinline__ T sel3(T v0, T v1, T v2, int k) { return k == 0 ? v0 : (k == 1 ? v1 : v2); }

// Visit every tile whose cell-centre box, grown by R, meets the segment a -> b; only the slabs
// (layers of tiles across the ray's dominant axis) first, first + step, ... of them, so that
// `step` threads can share one ray. The reciprocals 1 / d are formed once per ray.
template <typename F>
__device__ __forceinline__ void for_each_tile(const BinGeom& g, float bx, float by, float bz, F f, int first = 0,
                                              int step = 1) {
    const float a[3] = {g.ax, g.ay, g.az};
    const float d[3] = {bx - g.ax, by - g.ay, bz - g.az};
    float inv[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) inv[k] = d[k] != 0.0f ? 1.0f / d[k] : 0.0f;
    const float glo[3] = {-g.R, -g.R, -g.R};
    const float ghi[3] = {(float)(g.G - 1) + g.R, (float)(g.G - 1) + g.R, (float)(g.Gz - 1) + g.R};
    float t0 = 0.0f, t1 = 1.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (d[k] == 0.0f) {
            if (a[k] < glo[k] || a[k] > ghi[k]) return;
        } else {
            const float e0 = (glo[k] - a[k]) * inv[k], e1 = (ghi[k] - a[k]) * inv[k];
            t0 = fmaxf(t0, fminf(e0, e1));
            t1 = fminf(t1, fmaxf(e0, e1));
        }
    }
    if (t0 > t1) return;
    int A = 0;
    float dmax = fabsf(d[0]);
    if (fabsf(d[1]) > dmax) {
        A = 1;
        dmax = fabsf(d[1]);
    }
    if (fabsf(d[2]) > dmax) A = 2;
    const int Bx = (A + 1) % 3, Cx = (A + 2) % 3;
    // the dominant axis A and the two others, B and C
    const float aA = sel3(a[0], a[1], a[2], A), dA = sel3(d[0], d[1], d[2], A), invA = sel3(inv[0], inv[1], inv[2], A);
    const float aB = sel3(a[0], a[1], a[2], Bx), dB = sel3(d[0], d[1], d[2], Bx);
    const float aC = sel3(a[0], a[1], a[2], Cx), dC = sel3(d[0], d[1], d[2], Cx);
    const int tsA = sel3(g.tx, g.ty, g.tz, A), tsB = sel3(g.tx, g.ty, g.tz, Bx), tsC = sel3(g.tx, g.ty, g.tz, Cx);
    const int ntA = sel3(g.ntx, g.nty, g.ntz, A), ntB = sel3(g.ntx, g.nty, g.ntz, Bx);
    const int ntC = sel3(g.ntx, g.nty, g.ntz, Cx);
    const float pa0 = aA + dA * t0, pa1 = aA + dA * t1;
    int ta0 = (int)floorf((fminf(pa0, pa1) - g.R) / (float)tsA);
    int ta1 = (int)floorf((fmaxf(pa0, pa1) + g.R) / (float)tsA);
    ta0 = max(ta0, 0);
    ta1 = min(ta1, ntA - 1);
    for (int ta = ta0 + first; ta <= ta1; ta += step) {
        const float slo = (float)(ta * tsA) - g.R, shi = (float)(ta * tsA + tsA - 1) + g.R;
        float s0 = t0, s1 = t1;
        if (dA != 0.0f) {
            const float e0 = (slo - aA) * invA, e1 = (shi - aA) * invA;
            s0 = fmaxf(s0, fminf(e0, e1));
            s1 = fminf(s1, fmaxf(e0, e1));
        } else if (aA < slo || aA > shi) {
            continue;
        }
        if (s0 > s1) continue;
        const float b0 = aB + dB * s0, b1 = aB + dB * s1;
        const float c0 = aC + dC * s0, c1 = aC + dC * s1;
        int tb0 = max((int)floorf((fminf(b0, b1) - g.R) / (float)tsB), 0);
        int tb1 = min((int)floorf((fmaxf(b0, b1) + g.R) / (float)tsB), ntB - 1);
        int tc0 = max((int)floorf((fminf(c0, c1) - g.R) / (float)tsC), 0);
        int tc1 = min((int)floorf((fmaxf(c0, c1) + g.R) / (float)tsC), ntC - 1);
        for (int tb = tb0; tb <= tb1; ++tb) {
            for (int tc = tc0; tc <= tc1; ++tc) {
                // the tile's (x, y, z) index: ta along A, tb along B, tc along C
                const int tx = A == 0 ? ta : (Bx == 0 ? tb : tc);
                const int ty = A == 1 ? ta : (Bx == 1 ? tb : tc);
                const int tz = A == 2 ? ta : (Bx == 2 ? tb : tc);
                const float l[3] = {(float)(tx * g.tx) - g.R, (float)(ty * g.ty) - g.R, (float)(tz * g.tz) - g.R};
                const float h[3] = {(float)(tx * g.tx + g.tx - 1) + g.R, (float)(ty * g.ty + g.ty - 1) + g.R,
                                    (float)(tz * g.tz + g.tz - 1) + g.R};
                if (seg_box(a, d, inv, l, h, t0, t1)) f(tx + g.ntx * (ty + g.nty * tz));
            }
        }
    }
}

// The sensor's place in cell-index space comes from the frame scalars in device memory, so a
// captured graph stays valid while the sensor moves.
__device__ __forceinline__ void place_sensor(BinGeom& g, const DevParams& p, const FrameParams& f) {
    const float hg = (float)p.G / 2.0f, hz = (float)p.Gz / 2.0f;
    // a point q (metres, sensor frame) sits at u = (q + s)/res + G/2 - 0.5
    g.ax = f.sensor_x / p.res + hg - 0.5f;
    g.ay = f.sensor_y / p.res + hg - 0.5f;
    g.az = f.sensor_z / p.res + hz - 0.5f;
}

struct RayPrep {
    bool ok;
    float bx, by, bz;  // far end of the binned segment (cell-index space)
};

// Per-ray constants. K3DOM: (m, d_m) and (m/d_m, margin), d_m and margin as the reference
// forms them (mass_update.cu:29-31,55). DS: (m, |m|^2) as measurement_grid.cu:90.
// consts = false: only ok and the segment's far end (K3DOM), for a second thread of the ray.
__device__ __forceinline__ RayPrep prep_ray(const DevParams& p, const BinGeom& g, float mx, float my, float mz,
                                           bool ds, float4* ra, double4* rc, bool consts = true) {
    RayPrep r;
    r.ok = isfinite(mx) && isfinite(my) && isfinite(mz);
    r.bx = r.by = r.bz = 0.0f;
    *ra = make_float4(0.f, 0.f, 0.f, 0.f);
    *rc = make_double4(0.0, 0.0, 0.0, 0.0);
    if (!r.ok) return r;
    const float sq = __fadd_rn(__fadd_rn(__fmul_rn(mx, mx), __fmul_rn(my, my)), __fmul_rn(mz, mz));
    if (!ds && !consts) {
        r.bx = g.ax + mx / p.res;
        r.by = g.ay + my / p.res;
        r.bz = g.az + mz / p.res;
    } else if (!ds) {
        // d_m and the margin point (mass_update.cu:29-31,55) in FP64; a zero-length ray gets
        // 1/d_m = 0, which turns its free evidence off as the reference's NaN comparisons do
        const double dmd = sqrt((double)mx * mx + (double)my * my + (double)mz * mz);
        const double margd = fmax(0.9 * dmd, dmd - 2.0 * (double)p.res);
        const double inv = dmd > 0.0 ? 1.0 / dmd : 0.0;
        const float dm = (float)dmd;
        *ra = make_float4(mx, my, mz, dm);
        *rc = make_double4(dmd, margd, inv, 0.0);
        r.bx = g.ax + mx / p.res;
        r.by = g.ay + my / p.res;
        r.bz = g.az + mz / p.res;
    } else {
        *ra = make_float4(mx, my, mz, sq);
        const float len = sqrtf(sq);
        if (!(len > 0.0f)) {
            r.ok = false;  // |m| = 0: inner product 0, never a neighbour (measurement_grid.cu:92)
            return r;
        }
        const float L = sqrtf((float)(2 * g.G * g.G + g.Gz * g.Gz)) + 2.0f * g.R + 4.0f;  // cells
        const float sc = L / (len / p.res);
        r.bx = g.ax + mx / p.res * sc;
        r.by = g.ay + my / p.res * sc;
        r.bz = g.az + mz / p.res * sc;
    }
    return r;
}


__device__ __forceinline__ BinGeom scene_geom(const SceneDev& sd, const FrameParams& f) {
    BinGeom g;
    g.R = sd.bin_R;
    g.G = sd.p.G;
    g.Gz = sd.p.Gz;
    g.tx = sd.ts.tx; g.ty = sd.ts.ty; g.tz = sd.ts.tz;
    g.ntx = sd.ts.ntx; g.nty = sd.ts.nty; g.ntz = sd.ts.ntz;
    place_sensor(g, sd.p, f);
    return g;
}

// Pass 1 over every point slot of every scene: per-ray constants and the number of tiles the
// ray's support reaches (0 for slots past the scene's point count). TALLY (placed lists): each
// reached tile's ray count is also added to tile_tally, through a block histogram of the T tiles
// in shared memory (the tiles around a sensor are reached by nearly every ray: one global atomic
// per block and tile instead of one per ray); the value that atomic returns is the block's first
// slot in the tile's range (relative to its start), kept in block_base for k_ray_place. TALLY
// also gives each ray two threads (the ray's even and odd slabs of tiles, counts per thread):
// the walk is latency bound, and 120,000 rays make only 25 warps per SM.
template <bool TALLY>
__global__ void k_ray_count(Batch bt, const float* __restrict__ xs, const float* __restrict__ ys,
                            const float* __restrict__ zs, int ds, float4* __restrict__ ra,
                            double4* __restrict__ rc, uint32_t* __restrict__ counts,
                            uint32_t* __restrict__ tile_tally, uint32_t* __restrict__ block_base,
                            DevStatus* status) {
    extern __shared__ uint32_t s_tally[];  // [T] (TALLY)
    if (blockIdx.x == 0 && threadIdx.x == 0) status->overflow = 0u;  // per-frame flag (set by k_ray_emit / k_tile_ranges)
    if (TALLY) {
        for (int t = threadIdx.x; t < bt.T; t += blockDim.x) s_tally[t] = 0u;
        __syncthreads();
    }
    constexpr int kPer = TALLY ? kRayThreads : 1;  // threads per ray
    const long nt = (long)bt.N * kPer;
    for (long tid = (long)blockIdx.x * blockDim.x + threadIdx.x; tid < nt; tid += (long)gridDim.x * blockDim.x) {
        const int i = (int)(tid / kPer), half = (int)(tid % kPer);
        const int sc = scene_of(bt.off->point, bt.S, i);
        const FrameParams f = bt.fp[sc];
        if (i - bt.off->point[sc] >= f.n_points) {
            counts[tid] = 0;
            continue;
        }
        const SceneDev& sd = bt.sc[sc];
        const BinGeom g = scene_geom(sd, f);
        float mx = xs[i], my = ys[i], mz = zs[i];
        if (f.has_transform) apply_transform(f, &mx, &my, &mz);
        float4 a;
        double4 cc;
        const RayPrep r = prep_ray(sd.p, g, mx, my, mz, ds != 0, &a, &cc, half == 0);
        if (half == 0) {
            ra[i] = a;
            rc[i] = cc;
        }
        uint32_t c = 0;
        if (r.ok) {
            const uint32_t toff = (uint32_t)bt.off->tile[sc];
            for_each_tile(
                g, r.bx, r.by, r.bz,
                [&](int t) {
                    ++c;
                    if (TALLY) atomicAdd(&s_tally[toff + (uint32_t)t], 1u);
                },
                half, kPer);
        } else if (half == 0 && !(isfinite(mx) && isfinite(my) && isfinite(mz))) {
            atomicAdd(&status->nonfinite_points, 1ull);
        }
        counts[tid] = c;
    }
    if (TALLY) {
        __syncthreads();
        uint32_t* row = block_base + (size_t)blockIdx.x * bt.T;
        for (int t = threadIdx.x; t < bt.T; t += blockDim.x) {
            const uint32_t v = s_tally[t];
            if (v) row[t] = atomicAdd(&tile_tally[t], v);
        }
    }
}

// Pass 2: (global tile, ray) entries at the ray's scanned offset.
__global__ void k_ray_emit(Batch bt, const float* __restrict__ xs, const float* __restrict__ ys,
                           const float* __restrict__ zs, int ds, const uint32_t* __restrict__ offsets,
                           uint32_t* __restrict__ total, long capacity, uint32_t* __restrict__ ekeys,
                           uint32_t* __restrict__ evals, DevStatus* status) {
    const bool over = (long)total[0] > capacity;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        total[2] = over ? 0u : total[0];  // live entry count for the sort
        if (over) atomicOr(&status->overflow, 1u);
    }
    if (over) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < bt.N; i += gridDim.x * blockDim.x) {
        const int sc = scene_of(bt.off->point, bt.S, i);
        const FrameParams f = bt.fp[sc];
        if (i - bt.off->point[sc] >= f.n_points) continue;
        const SceneDev& sd = bt.sc[sc];
        const BinGeom g = scene_geom(sd, f);
        float mx = xs[i], my = ys[i], mz = zs[i];
        if (f.has_transform) apply_transform(f, &mx, &my, &mz);
        float4 a;
        double4 c;
        const RayPrep r = prep_ray(sd.p, g, mx, my, mz, ds != 0, &a, &c);
        if (!r.ok) continue;
        // never write more entries than were counted: the count pass sized this ray's range
        const uint32_t o0 = offsets[i];
        const uint32_t cnt = (i + 1 < bt.N) ? offsets[i + 1] - o0 : total[0] - o0;
        const uint32_t toff = (uint32_t)bt.off->tile[sc];
        uint32_t o = o0;
        for_each_tile(g, r.bx, r.by, r.bz, [&](int t) {
            if (o - o0 < cnt) {
                ekeys[o] = toff + (uint32_t)t;
                evals[o] = (uint32_t)i;
                ++o;
            }
        });
        for (; o - o0 < cnt; ++o) {  // pad with a key past the last tile (sorted last, ignored)
            ekeys[o] = (uint32_t)bt.T;
            evals[o] = (uint32_t)i;
        }
    }
}

// tile_start[t] = first sorted entry of tile t, for t in [0, T].
__global__ void k_tile_start(const uint32_t* __restrict__ skeys, const uint32_t* __restrict__ total, int T,
                             uint32_t* __restrict__ tile_start) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t > T) return;
    const long n = (long)total[2];
    long lo = 0, hi = n;
    while (lo < hi) {
        const long mid = (lo + hi) >> 1;
        if (skeys[mid] < (uint32_t)t) lo = mid + 1; else hi = mid;
    }
    tile_start[t] = (uint32_t)lo;
}

__global__ void k_tile_items(const uint32_t* __restrict__ tile_start, int T, int chunk, uint32_t* __restrict__ items) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T) return;
    const uint32_t len = tile_start[t + 1] - tile_start[t];
    items[t] = len == 0 ? 1u : (len + chunk - 1) / chunk;
}

__global__ void k_finish_lists(const uint32_t* __restrict__ item_off, int T, DevStatus* status,
                               const uint32_t* __restrict__ total) {
    status->work_items = item_off[T];
    status->ray_entries = total[0];
    // k_ray_count has finished counting this frame's non-finite points: keep the frame's count
    status->nonfinite_frame = (unsigned int)status->nonfinite_points;
    status->nonfinite_points = 0;
    status->work_counter = 0;
    status->work_counter2 = 0;
    status->kernel_evals = 0;
}

// K3DOM lists without a sort. The evidence sums are exact integers, so the order of a tile's
// rays changes no result; k_ray_count<true> has tallied each tile's rays, this pass turns the
// tallies into ranges (tile_start) and clears them for the
// next frame, counts the work items per tile and their offsets, and ends the frame's list
// counters as k_finish_lists does. One block: a batch holds at most a few tens of thousands of
// tiles. On overflow (more entries than the list holds) every range is empty.
constexpr int kRangeThreads = 1024;
__global__ void __launch_bounds__(kRangeThreads)
    k_tile_ranges(uint32_t* __restrict__ tile_tally, int T, int chunk, long capacity, uint32_t* __restrict__ tile_start,
                  uint32_t* __restrict__ item_off, uint32_t* __restrict__ total, DevStatus* status) {
    __shared__ unsigned long long sm[kRangeThreads / 32 + 1];
    const int per = (T + kRangeThreads - 1) / kRangeThreads;
    const int t0 = min(T, (int)threadIdx.x * per), t1 = min(T, t0 + per);
    unsigned long long n = 0;
    for (int t = t0; t < t1; ++t) n += tile_tally[t];
    unsigned long long entries;
    const unsigned long long base = block_exclusive_scan<unsigned long long, kRangeThreads>(n, sm, &entries);
    const bool over = entries > (unsigned long long)capacity;
    unsigned long long o = over ? 0ull : base;
    unsigned long long ni = 0;
    for (int t = t0; t < t1; ++t) {
        const uint32_t c = over ? 0u : tile_tally[t];
        tile_start[t] = (uint32_t)o;
        o += c;
        ni += c == 0 ? 1u : (c + chunk - 1) / chunk;
    }
    unsigned long long items;
    const unsigned long long ibase = block_exclusive_scan<unsigned long long, kRangeThreads>(ni, sm, &items);
    unsigned long long io = ibase;
    for (int t = t0; t < t1; ++t) {
        const uint32_t c = over ? 0u : tile_tally[t];
        item_off[t] = (uint32_t)io;
        io += c == 0 ? 1u : (c + chunk - 1) / chunk;
        tile_tally[t] = 0u;
    }
    if (threadIdx.x == 0) {
        const uint32_t e32 = (uint32_t)min(entries, 0xFFFFFFFFull);
        tile_start[T] = over ? 0u : e32;
        item_off[T] = (uint32_t)items;
        total[0] = e32;
        total[2] = over ? 0u : e32;
        if (over) atomicOr(&status->overflow, 1u);
        status->work_items = (uint32_t)items;
        status->ray_entries = e32;
        // k_ray_count has finished counting this frame's non-finite points: keep the frame's count
        status->nonfinite_frame = (unsigned int)status->nonfinite_points;
        status->nonfinite_points = 0;
        status->work_counter = 0;
        status->work_counter2 = 0;
        status->kernel_evals = 0;
    }
}

// Pass 2 of the placed lists, on the grid of the tally (the same rays in each block): each ray
// takes one slot in the range of each tile it reaches, at most as many tiles as it tallied (the
// same enumeration as the tally's, on the same values), from the block's own share of the range,
// and never a slot past the list. The segment's far end is formed from the staged ray constants
// as prep_ray forms it.
template <typename F>
__device__ __forceinline__ void for_each_placed_tile(const Batch& bt, const float4* __restrict__ ra,
                                                     const uint32_t* __restrict__ counts, F f) {
    const long nt = (long)bt.N * kRayThreads;
    for (long tid = (long)blockIdx.x * blockDim.x + threadIdx.x; tid < nt; tid += (long)gridDim.x * blockDim.x) {
        const int i = (int)(tid / kRayThreads), half = (int)(tid % kRayThreads);
        const uint32_t cnt = counts[tid];
        if (cnt == 0u) continue;
        const int sc = scene_of(bt.off->point, bt.S, i);
        const SceneDev& sd = bt.sc[sc];
        const BinGeom g = scene_geom(sd, bt.fp[sc]);
        const float4 a = ra[i];
        const float bx = g.ax + a.x / sd.p.res, by = g.ay + a.y / sd.p.res, bz = g.az + a.z / sd.p.res;
        const uint32_t toff = (uint32_t)bt.off->tile[sc];
        uint32_t k = 0;
        for_each_tile(
            g, bx, by, bz,
            [&](int t) {
                if (k < cnt) {
                    f(i, toff + (uint32_t)t);
                    ++k;
                }
            },
            half, kRayThreads);
    }
}

__global__ void k_ray_place(Batch bt, const float4* __restrict__ ra, const uint32_t* __restrict__ counts,
                            const uint32_t* __restrict__ tile_start, const uint32_t* __restrict__ block_base,
                            const uint32_t* __restrict__ total, uint32_t* __restrict__ evals) {
    extern __shared__ uint32_t s_slot[];  // [T]: the block's next slot in each tile's range
    const uint32_t n = total[2];
    if (n == 0u) return;  // overflow, or no entries (the same for every thread)
    const uint32_t* row = block_base + (size_t)blockIdx.x * bt.T;
    // rows of tiles this block does not reach hold stale values that are never used
    for (int t = threadIdx.x; t < bt.T; t += blockDim.x) s_slot[t] = tile_start[t] + row[t];
    __syncthreads();
    for_each_placed_tile(bt, ra, counts, [&](int i, uint32_t gt) {
        const uint32_t pos = atomicAdd(&s_slot[gt], 1u);
        if (pos < n) evals[pos] = (uint32_t)i;
    });
}

// Blocks of the two placed-list passes (the same grid for both): at most kBinBlocksMax rows of
// block_base.
int bin_blocks(long n) { return (int)std::max(1L, std::min((n + kBlock - 1) / kBlock, (long)kBinBlocksMax)); }

// Largest |c| of a cell centre seen from a sensor inside or near the grid [m].
static float max_extent(const DevParams& p) { return 2.0f * ((float)p.G * p.res * 1.7320508f + p.size_z); }

void fill_scene_evidence(SceneDev& sd, bool ds, float4* ktab) {
    const DevParams& p = sd.p;
    if (!ds) {
        sd.bin_R = p.ls / p.res * (1.0f + 1e-4f) + 1e-3f;
    } else {
        // window radius plus the FP32 rounding slack of |c|^2 - (c.m)^2/|m|^2
        const float ext = max_extent(p);
        const float slack = 64.0f * 5.96e-8f * ext * ext;
        sd.bin_R = sqrtf(p.window_radius * p.window_radius + slack) / p.res + 1e-3f;
    }
    sd.wr2 = p.window_radius * p.window_radius;
    // cull around the sub-block centroid: half diagonal sqrt(1.5^2+1.5^2+0.5^2) res
    const float rsb = 2.1794495f * p.res;
    float rsup;
    if (!ds) {
        rsup = p.ls * (1.0f + 1e-4f) + rsb + 1e-3f * p.res;
    } else {
        const float ext = max_extent(p);
        const float slack = 64.0f * 5.96e-8f * ext * ext;
        rsup = sqrtf(p.window_radius * p.window_radius + slack) + rsb + 1e-3f * p.res;
    }
    sd.cull_r2 = rsup * rsup;
    // box culls (stage_pair, k_dsgrid): the support radius, or the DS window with the FP32 slack
    // of the reference's neighbour test, plus the same margin as rsup
    float rls;
    if (!ds) {
        rls = p.ls * (1.0f + 1e-4f) + 1e-3f * p.res;
    } else {
        const float ext = max_extent(p);
        const float slack = 64.0f * 5.96e-8f * ext * ext;
        rls = sqrtf(p.window_radius * p.window_radius + slack) + 1e-3f * p.res;
    }
    sd.cull_ls2 = rls * rls;
    // fixed point: one kernel value is at most sigma -> at most 2^40 units, leaving 2^23 terms
    // of headroom in a signed 64-bit sum
    const double sig = std::max((double)p.sigma, 1e-30);
    const int sh = 40 - (int)std::ceil(std::log2(sig));
    sd.fx_inv = std::ldexp(1.0, -sh);
    if (ktab) build_kernel_table(p.sigma, std::ldexp(1.0, sh), ktab);
}

// Worst case of tiles one ray can reach: for each slab of tiles along the ray's dominant axis A,
// the segment clipped to the slab grown by R spans at most ts[A] - 1 + 2R cells along every
// axis (|d_o| <= |d_A|), and the tiles within R of it along axis o number at most
// ceil((ts[A] + 4R) / ts[o]) + 1. Times the slabs, for the worst axis.
long ray_entries_bound(const DevParams& p, const TileShape& ts, int max_points, float bin_R) {
    const double R = (double)bin_R + 0.01;
    const int tsz[3] = {ts.tx, ts.ty, ts.tz}, nt[3] = {ts.ntx, ts.nty, ts.ntz};
    long worst = 0;
    for (int A = 0; A < 3; ++A) {
        long per_slab = 1;
        for (int k = 1; k <= 2; ++k) {
            const int o = (A + k) % 3;
            const long n = (long)std::ceil((tsz[A] + 4.0 * R) / tsz[o]) + 1;
            per_slab *= std::min<long>(n, nt[o]);
        }
        worst = std::max(worst, per_slab * nt[A]);
    }
    worst = std::min<long>(worst, (long)ts.ntx * ts.nty * ts.ntz);
    return worst * (long)max_points;
}

cudaError_t build_ray_lists(const Batch& bt, const float* xs, const float* ys, const float* zs, RayBuffers& rb,
                            bool ds, DevStatus* status, const SortWait& wait, cudaStream_t st) {
    const int N = bt.N;
    const int T = bt.T;
    if (placed_lists(ds, T)) {  // K3DOM: tally, ranges, place
        const size_t hist = sizeof(uint32_t) * (size_t)T;
        const int blocks = bin_blocks((long)N * kRayThreads);
        ++g_launches;
        k_ray_count<true><<<blocks, kBlock, hist, st>>>(bt, xs, ys, zs, 0, rb.ray_a, rb.ray_c, rb.counts,
                                                         rb.tile_tally, rb.block_base, status);
        ++g_launches;
        k_tile_ranges<<<1, kRangeThreads, 0, st>>>(rb.tile_tally, T, rb.chunk, rb.capacity, rb.tile_start,
                                                   rb.item_off, rb.total, status);
        ++g_launches;
        k_ray_place<<<blocks, kBlock, hist, st>>>(bt, rb.ray_a, rb.counts, rb.tile_start, rb.block_base, rb.total,
                                                   rb.evals2);
        return cudaGetLastError();
    }
    // DS (and batches with more tiles than a block histogram holds): entries in ray order, then a
    // stable sort by tile
    ++g_launches;
    k_ray_count<false><<<grid_for(N), kBlock, 0, st>>>(bt, xs, ys, zs, ds ? 1 : 0, rb.ray_a, rb.ray_c, rb.counts,
                                                        nullptr, nullptr, status);
    cudaError_t e = scan_u32_exclusive(rb.counts, rb.offsets, N, rb.scan_tmp, rb.total, st);
    if (e != cudaSuccess) return e;
    ++g_launches;
    k_ray_emit<<<grid_for(N), kBlock, 0, st>>>(bt, xs, ys, zs, ds ? 1 : 0, rb.offsets, rb.total, rb.capacity,
                                               rb.ekeys, rb.evals, status);
    int bits = 1;
    while ((1 << bits) < T + 1) ++bits;
    // stable: each tile keeps its rays in input order (the DS first-100 rule depends on it)
    SortWait w = wait;
    w.skip_tile = -1;
    e = onesweep_sort_pairs_dn(rb.ekeys, rb.evals, rb.ekeys2, rb.evals2, rb.ekeys_alt, rb.evals_alt, rb.capacity,
                               rb.total + 2, bits, rb.os_scratch, rb.os_words, status, w, st);
    if (e != cudaSuccess) return e;
    ++g_launches;
    k_tile_start<<<div_up(T + 1, kBlock), kBlock, 0, st>>>(rb.ekeys2, rb.total, T, rb.tile_start);
    ++g_launches;
    k_tile_items<<<div_up(T, kBlock), kBlock, 0, st>>>(rb.tile_start, T, rb.chunk, rb.tile_items);
    e = scan_u32_exclusive(rb.tile_items, rb.item_off, T, rb.scan_tmp, rb.item_off + T, st);
    if (e != cudaSuccess) return e;
    ++g_launches;
    k_finish_lists<<<1, 1, 0, st>>>(rb.item_off, T, status, rb.total);
    return cudaGetLastError();
}

// ================================================================ shared kernel machinery
__device__ __forceinline__ int find_tile(const uint32_t* __restrict__ item_off, int T, uint32_t item) {
    // last t with item_off[t] <= item
    int lo = 0, hi = T;  // answer in [0, T)
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (item_off[mid] <= item) lo = mid; else hi = mid;
    }
    return lo;
}

struct CellLoc {
    int c;          // cell index within the scene, -1 when outside the grid
    int local;      // cell index within the tile
    float x, y, z;  // cell centre relative to the sensor [m], reference FP32 operation order
    float ox, oy, oz;  // anchor: centre of the sub-block's cell (2, 2, 1), same formula
};

// Cell centre of index triple (ix, iy, iz), the expression of mass_update.cu:92-99 /
// measurement_grid.cu:77-84 evaluated in FP32 in the reference's order.
__device__ __forceinline__ void centre_xyz(int ix, int iy, int iz, const DevParams& p, float sx, float sy, float sz,
                                           float* x, float* y, float* z) {
    const float hg = __fdiv_rn((float)p.G, 2.0f), hz = __fdiv_rn((float)p.Gz, 2.0f);
    *x = __fsub_rn(__fmul_rn(__fsub_rn(__fadd_rn((float)ix, 0.5f), hg), p.res), sx);
    *y = __fsub_rn(__fmul_rn(__fsub_rn(__fadd_rn((float)iy, 0.5f), hg), p.res), sy);
    *z = __fsub_rn(__fmul_rn(__fsub_rn(__fadd_rn((float)iz, 0.5f), hz), p.res), sz);
}

__device__ __forceinline__ CellLoc locate(const DevParams& p, const TileShape& ts, int t, int sb, int lane,
                                          float sx, float sy, float sz) {
    const int tx = t % ts.ntx, ty = (t / ts.ntx) % ts.nty, tz = t / (ts.ntx * ts.nty);
    const int sbx = sb % ts.nsbx, sby = (sb / ts.nsbx) % ts.nsby, sbz = sb / (ts.nsbx * ts.nsby);
    const int lx = sbx * 4 + (lane & 3), ly = sby * 4 + ((lane >> 2) & 3), lz = sbz * 2 + (lane >> 4);
    const int ix = tx * ts.tx + lx, iy = ty * ts.ty + ly, iz = tz * ts.tz + lz;
    CellLoc L;
    L.local = lx + ts.tx * (ly + ts.ty * lz);
    const bool in = ix < p.G && iy < p.G && iz < p.Gz;
    L.c = in ? ix + p.G * iy + p.G * p.G * iz : -1;
    centre_xyz(ix, iy, iz, p, sx, sy, sz, &L.x, &L.y, &L.z);
    centre_xyz(tx * ts.tx + sbx * 4 + 2, ty * ts.ty + sby * 4 + 2, tz * ts.tz + sbz * 2 + 1, p, sx, sy, sz, &L.ox,
               &L.oy, &L.oz);
    return L;
}

// Sub-blocks go to the warps nearest to the sensor first. A sub-block's work grows with the rays
// that pass it, which is largest on the tile's sensor side (rays that end inside the tile never
// reach its far side, and near the sensor every ray passes close), so the costly sub-blocks start
// first and the cheap ones fill the end of the work item, where warps that run out of sub-blocks
// wait at the item's barrier. The sums are exact, so the order changes no result.
constexpr int kMaxOrderedSb = 64;  // the largest tiling (16x16x8) has 64 sub-blocks

struct SbOrder {
    float key[kMaxOrderedSb];
    uint8_t idx[kMaxOrderedSb];
};

// Phase 1 (thread i < nsb): squared distance of sub-block i's anchor from the sensor.
__device__ __forceinline__ void sb_order_keys(SbOrder& o, const DevParams& p, const TileShape& ts, int t, int nsb,
                                              float sx, float sy, float sz) {
    const int i = threadIdx.x;
    if (nsb > kMaxOrderedSb || i >= nsb) return;
    const int tx = t % ts.ntx, ty = (t / ts.ntx) % ts.nty, tz = t / (ts.ntx * ts.nty);
    const int sbx = i % ts.nsbx, sby = (i / ts.nsbx) % ts.nsby, sbz = i / (ts.nsbx * ts.nsby);
    float x, y, z;
    centre_xyz(tx * ts.tx + sbx * 4 + 2, ty * ts.ty + sby * 4 + 2, tz * ts.tz + sbz * 2 + 1, p, sx, sy, sz, &x, &y, &z);
    o.key[i] = x * x + y * y + z * z;
}

// Phase 2, after a barrier: sub-block i's place in the order (ties by index).
__device__ __forceinline__ void sb_order_rank(SbOrder& o, int nsb) {
    const int i = threadIdx.x;
    if (nsb > kMaxOrderedSb || i >= nsb) return;
    const float k = o.key[i];
    int r = 0;
    for (int j = 0; j < nsb; ++j) {
        const float kj = o.key[j];
        r += (kj < k) || (kj == k && j < i);
    }
    o.idx[r] = (uint8_t)i;
}

__device__ __forceinline__ int sb_at(const SbOrder& o, int n, int nsb) { return nsb > kMaxOrderedSb ? n : o.idx[n]; }

// The work item a CTA holds: its tile (global and scene-local), scene and ray range.
struct Item {
    int t, lt, sc;
    uint32_t k, n_items, e0;
    int nr;
};

__device__ __forceinline__ Item item_of(const Batch& bt, const uint32_t* item_off, const uint32_t* tile_start,
                                        uint32_t item, int chunk) {
    Item it;
    it.t = find_tile(item_off, bt.T, item);
    it.sc = scene_of(bt.off->tile, bt.S, it.t);
    it.lt = it.t - bt.off->tile[it.sc];
    it.k = item - item_off[it.t];
    it.n_items = item_off[it.t + 1] - item_off[it.t];
    it.e0 = tile_start[it.t] + it.k * (uint32_t)chunk;
    const uint32_t e1 = min(tile_start[it.t + 1], it.e0 + (uint32_t)chunk);
    it.nr = (int)(e1 > it.e0 ? e1 - it.e0 : 0);
    return it;
}

struct EvArgs {
    Batch bt;
    const uint32_t* item_off;
    const uint32_t* tile_start;
    const uint32_t* evals;
    const float4* ray_a;
    const double4* ray_c;
    const float4* ktab;  // S tables of kKernelTab entries, fixed-point scale folded in
    uint32_t* tile_done;
    unsigned long long* acc;
    uint8_t* ds_counts;
    long ds_count_capacity;
    CellState cs;
    CellWork cw;
    DevStatus* status;
    int first_frame;
    int chunk;  // rays per work item (<= kChunk)
    int fuse_update;  // K3DOM: the last CTA of a tile updates its cells (else k_k3dom_update_cells)
    cudaTextureObject_t ktex;  // ktab through the texture path
};

// ================================================================ K3DOM
// The sparse kernel of mass_update.cu:24-26,
//   k(d) = max(0, sigma ((2 + cos(2 pi x)) (1 - x) / 3 + sin(2 pi x) / (2 * 3.141592))),  x = d / ls,
// (the reference's truncated pi in the sine term is kept) is tabulated as a function of
// u = d^2 / ls^2 (no square root in the hot loop): kKernelTab intervals, on each a cubic in the
// local coordinate through four FP64 samples (f = 0, 1/3, 2/3, 1). Evaluated in FP32 by Horner,
// it is within 1.2e-7 relative of the FP64 kernel wherever k > 1e-3 sigma and within 8e-8 sigma
// absolute everywhere; the direct FP32 formula loses up to ~1e-5 to cancellation between its two
// terms over the outer half of the support.
static double kernel_ref(double u, double sigma) {
    const double x = std::sqrt(u);
    const double v = sigma * ((2.0 + std::cos(M_PI * 2.0 * x)) * (1.0 - x) / 3.0 +
                              std::sin(M_PI * 2.0 * x) / (2.0 * 3.141592));
    return v > 0.0 ? v : 0.0;
}

void build_kernel_table(float sigma, double scale, float4* out) {
    for (int i = 0; i < kKernelTab; ++i) {
        double y[4];
        for (int j = 0; j < 4; ++j) y[j] = scale * kernel_ref(std::min(1.0, (i + j / 3.0) / kKernelTab), sigma);
        // inverse Vandermonde of the nodes 0, 1/3, 2/3, 1
        const double c0 = y[0];
        const double c1 = -5.5 * y[0] + 9.0 * y[1] - 4.5 * y[2] + y[3];
        const double c2 = 9.0 * y[0] - 22.5 * y[1] + 18.0 * y[2] - 4.5 * y[3];
        const double c3 = -4.5 * y[0] + 13.5 * y[1] - 13.5 * y[2] + 4.5 * y[3];
        out[i] = make_float4((float)c0, (float)c1, (float)c2, (float)c3);
    }
    out[kKernelTab] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// Table position t = d^2 * (kKernelTab / ls^2) = u * kKernelTab (the factor kKernelTab is a power
// of two, so folding it into 1 / ls^2 changes no bit): interval i = floor(t), offset f = t - i.
// Inside the support (d^2 < ls^2) t <= kKernelTab, and entry kKernelTab is zero, so no clamp is
// needed. The floor is taken without conversion instructions: t + 2^23 rounded down is
// 2^23 + floor(t) exactly for 0 <= t < 2^23, whose low mantissa bits are floor(t).
struct TabPos {
    int i;
    float f;
};
__device__ __forceinline__ TabPos tab_pos(float t) {
    const float tr = __fadd_rd(t, 8388608.0f);
    TabPos q;
    q.i = __float_as_int(tr) - 0x4B000000;
    q.f = t - (tr - 8388608.0f);
    return q;
}
__device__ __forceinline__ float tab_eval(const float4* __restrict__ tab, TabPos q) {
    const float4 c = tab[q.i];
    return fmaf(q.f, fmaf(q.f, fmaf(q.f, c.w, c.z), c.y), c.x);
}
__device__ __forceinline__ float tab_eval_tex(cudaTextureObject_t tab, int base, TabPos q) {
    const float4 c = tex1Dfetch<float4>(tab, base + q.i);
    return fmaf(q.f, fmaf(q.f, fmaf(q.f, c.w, c.z), c.y), c.x);
}
__device__ __forceinline__ float kernel_tab(const float4* __restrict__ tab, float t) {
    return tab_eval(tab, tab_pos(t));
}

// mass_update.cu:12-14, 1 - 2 / (1 + exp(2 mass / mass_scale)), with k2 = 2 / mass_scale
__device__ __forceinline__ double calc_credit(double mass, double k2) {
    return 1.0 - 2.0 / (1.0 + exp(mass * k2));
}
__device__ __forceinline__ double positive_diff(double a, double b) { return fmax(0.0, a - b); }
// mass_update.cu:16-19, 1 / (1 + rest / numerator), written numerator / (numerator + rest)
__device__ __forceinline__ double calc_ratio(double numerator, double rest) {
    return (numerator <= 0.0 || rest < 0.0) ? 0.0 : numerator / (numerator + rest);
}
__device__ __forceinline__ float calc_norm(float weight_sum, float rho_p) {
    return weight_sum > 0.0f ? rho_p / weight_sum : 0.0f;
}

// gridCellPredictionUpdateKernel's per-cell body (mass_update.cu:163-181) plus the per-cell
// updates of the persistent-particle and moment stages. Masses are stored in FP32; the update
// is evaluated in FP64 (it has several cancelling differences) and rounded once.
// g = gamma^dt of the frame.
// A cell's inputs to the update, loaded together so that their reads overlap (the particle sums
// are read whether or not the cell holds particles; they are used only when it does).
struct CellIn {
    float m_f, m_s, m_d, sum_w, wvx, wvy, wvz;
    int start;
};
__device__ __forceinline__ CellIn load_cell_in(const CellState& cs, const CellWork& cw, int c, bool first_frame) {
    CellIn in;
    in.m_f = cs.free_m[c];
    in.m_s = cs.static_m[c];
    in.m_d = cs.dyn_m[c];
    in.start = first_frame ? -1 : cw.start[c];
    in.sum_w = cw.sum_w[c];
    in.wvx = cw.sum_wvx[c];
    in.wvy = cw.sum_wvy[c];
    in.wvz = cw.sum_wvz[c];
    return in;
}

// The update of cell c from its inputs `in` (outputs written to cs, cw).
__device__ void k3dom_cell_update_in(const DevParams& p, double g, int c, double del_occ, double del_free,
                                     const CellIn& in, CellState cs, CellWork cw, bool first_frame) {
    double m_f = in.m_f, m_s = in.m_s, m_d = in.m_d;
    const int start = in.start;
    const bool has = start >= 0;
    const double dyn_pred = has ? (double)in.sum_w : 0.0;
    const double k2 = 2.0 / (double)p.mass_scale;
    const double pred_total = (m_f + m_d) * g;
    // predict_mass (:79-84)
    m_s *= g;
    m_d = fmin(dyn_pred, fmax(0.0, pred_total - m_s));
    m_f = pred_total - m_d;
    // update_mass (:86-139)
    if (del_free > 0.0 || del_occ > 0.0) {
        const double del_sigma = del_free + del_occ;
        const double prime_sigma = m_f + m_s + m_d;
        double l_DtoF = 0.0, l_StoFD = 0.0, l_FtoD = 0.0;
        if (prime_sigma > 0.0) {
            // base_f m / prime_sigma with base_f = credit (del_free - del_occ)+ / del_sigma:
            // one reciprocal of z = del_sigma prime_sigma serves the three fractions
            const double z = del_sigma * prime_sigma;
            const double w = calc_credit(sqrt(z), k2) / z;
            const double wf = w * positive_diff(del_free, del_occ);
            const double wo = w * positive_diff(del_occ, del_free);
            l_DtoF = wf * m_d;
            l_StoFD = wf * positive_diff(m_s + m_d, m_f);
            l_FtoD = wo * positive_diff(m_f, m_s + m_d);
        }
        const double diff_f = l_StoFD / 2.0 * m_s + l_DtoF * m_d - l_FtoD * m_f;
        const double diff_s = -l_StoFD * m_s;
        const double diff_d = l_FtoD * m_f + l_StoFD / 2.0 * m_s - l_DtoF * m_d;
        m_f += diff_f;
        m_s += diff_s;
        m_d += diff_d;
        const double credit2 = calc_credit(m_s + m_d, k2);
        const double beta = (1.0 - credit2) + credit2 * calc_ratio(m_s, m_d);
        m_s = m_s + beta * del_occ;
        m_d = m_d + (1.0 - beta) * del_occ;
        m_f = m_f + del_free;
    }
    // separate_newborn_part (:141-150)
    double born;
    if (dyn_pred <= 0.0) born = m_d;
    else if (pred_total <= dyn_pred) born = 0.0;
    else born = (m_d * p.p_B * (pred_total - dyn_pred)) / (dyn_pred + p.p_B * (pred_total - dyn_pred));
    const double pers = m_d - born;
    cs.free_m[c] = (float)m_f;
    cs.static_m[c] = (float)m_s;
    cs.dyn_m[c] = (float)m_d;
    cs.born_m[c] = (float)born;
    cs.pers_m[c] = (float)pers;
    cs.pred_m[c] = (float)dyn_pred;
    cw.del_occ[c] = (float)del_occ;
    cw.del_free[c] = (float)del_free;
    if (first_frame) return;
    // updatePersistentParticlesKernel2: mu_UA = pers / pred (p_A = 0 -> the only factor)
    const double mu_UA = (has && dyn_pred > 0.0) ? pers / dyn_pred : 0.0;
    cw.factor[c] = (float)mu_UA;
    // statisticalMomentsKernel2 with sum(w' v) = mu_UA * sum(w v)
    double vx = 0.0, vy = 0.0, vz = 0.0;
    if (has && pers > 0.0) {
        const double q = mu_UA / pers;
        vx = q * (double)in.wvx;
        vy = q * (double)in.wvy;
        vz = q * (double)in.wvz;
    }
    cs.mvx[c] = (float)vx;
    cs.mvy[c] = (float)vy;
    cs.mvz[c] = (float)vz;
}

__device__ __forceinline__ void k3dom_cell_update(const DevParams& p, double g, int c, double del_occ,
                                                  double del_free, CellState cs, CellWork cw, bool first_frame) {
    k3dom_cell_update_in(p, g, c, del_occ, del_free, load_cell_in(cs, cw, c, first_frame), cs, cw, first_frame);
}

// Shared memory of k_bgki: one chunk of rays and a per-warp staging area for the FP64
// (sub-block, ray) constants of the rays that pass the cull. (The kernel table is read through
// the texture path: its lanes' scattered 16-byte reads ran 10 % slower from shared memory,
// where they conflicted on banks and queued behind the staging loads.)
// (dynamic, sized by the work item's ray count so that smaller chunks leave room for more CTAs)
struct BgkiSmem {
    float* stage;                 // [warps][kStageWarpFloats] pair records of the passing rays
    float4* a;                    // [chunk] m.x, m.y, m.z, d_m
    double4* c;                   // [chunk] d_m, margin, 1/d_m
    uint16_t* reg;                // [kRegions][chunk] rays per region of a 16x16 tile (region builds)
};

// A 16x16-cell tile splits into kRegions columns of 8x8 cells (full tile height); a ray's region
// list holds it when its segment meets the column's cell-centre box grown by the binning radius
// (plus a quarter cell), the test that put it in the tile's list, so every ray that can reach a
// cell of the column is in the column's list. Sub-blocks then cull only their column's rays.
constexpr int kRegions = 4;

// A pair record holds the staged constants of two rays a, b interleaved per component, so that one
// 8-byte register pair feeds a packed instruction:
//   float4 0: (perp0.x, perp0.y) of a, b     1: (perp0.z, par0)
//   float4 2: (u.x, u.y)                     3: (u.z, par0 - margin)
//   float4 4: (occ0.x, occ0.y)               5: (occ0.z, par0 - d_m)
// each float4 as (a, b, a, b); a seventh float4 pads the record so that the 32 lanes' scalar
// stores spread over the banks.
constexpr int kStagePairFloats = 28;
constexpr int kStageWarpFloats = 16 * kStagePairFloats;

__host__ __device__ constexpr size_t bgki_fixed_bytes(int warps) {
    return (sizeof(float) * (size_t)warps * kStageWarpFloats + 31) & ~(size_t)31;
}

inline size_t bgki_smem_bytes(int chunk, int warps = kEvWarps, bool regions = false) {
    return bgki_fixed_bytes(warps) + (size_t)chunk * (sizeof(float4) + sizeof(double4)) +
           (regions ? (size_t)kRegions * chunk * sizeof(uint16_t) : 0);
}

__device__ __forceinline__ BgkiSmem bgki_smem(unsigned char* base, int chunk, int warps) {
    BgkiSmem S;
    S.stage = reinterpret_cast<float*>(base);
    const size_t off = bgki_fixed_bytes(warps);
    S.c = reinterpret_cast<double4*>(base + off);  // 32-byte aligned
    S.a = reinterpret_cast<float4*>(base + off + sizeof(double4) * (size_t)chunk);
    S.reg = reinterpret_cast<uint16_t*>(base + off + (sizeof(double4) + sizeof(float4)) * (size_t)chunk);
    return S;
}

// Parameter interval [t0, t1] of a + t d inside the slab lo <= u <= hi (empty when t0 > t1).
__device__ __forceinline__ void slab(float a, float d, float lo, float hi, float* t0, float* t1) {
    if (d == 0.0f) {
        const bool in = a >= lo && a <= hi;
        *t0 = in ? -INFINITY : INFINITY;
        *t1 = in ? INFINITY : -INFINITY;
        return;
    }
    const float inv = 1.0f / d;
    const float e0 = (lo - a) * inv, e1 = (hi - a) * inv;
    *t0 = fminf(e0, e1);
    *t1 = fmaxf(e0, e1);
}

// Bit q (q = qx + 2 qy) set when the ray's binned segment a -> a + d (cell-index space) meets
// region q's box [x0 + 8 qx, x0 + 8 qx + 7] x [y0 + 8 qy, +7] x [z0, z0 + tz - 1] grown by R.
__device__ __forceinline__ unsigned region_mask(float ax, float ay, float az, float dx, float dy, float dz, float x0,
                                                float y0, float z0, int tz, float R) {
    float zl, zh;
    slab(az, dz, z0 - R, z0 + (float)(tz - 1) + R, &zl, &zh);
    zl = fmaxf(zl, 0.0f);
    zh = fminf(zh, 1.0f);
    float xl[2], xh[2], yl[2], yh[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        slab(ax, dx, x0 + 8.0f * h - R, x0 + 8.0f * h + 7.0f + R, &xl[h], &xh[h]);
        slab(ay, dy, y0 + 8.0f * h - R, y0 + 8.0f * h + 7.0f + R, &yl[h], &yh[h]);
    }
    unsigned q = 0;
#pragma unroll
    for (int qy = 0; qy < 2; ++qy)
#pragma unroll
        for (int qx = 0; qx < 2; ++qx)
            if (fmaxf(zl, fmaxf(xl[qx], yl[qy])) <= fminf(zh, fminf(xh[qx], yh[qy]))) q |= 1u << (qx + 2 * qy);
    return q;
}

// Stages the item's rays (m, d_m) and FP64 constants in shared memory and, for a 16x16 tile,
// appends each ray to the lists of the regions it reaches (rcnt zeroed before the call; list
// order is arbitrary, the sums are exact). Every thread of the block calls it.
template <int THREADS>
__device__ __forceinline__ void stage_item_rays(const EvArgs& A, const Item& it, const SceneDev& sd,
                                                const FrameParams& fp, bool regions, float4* sa, double4* sc,
                                                uint16_t* reg, int* rcnt) {
    const DevParams& p = sd.p;
    const TileShape& ts = sd.ts;
    const int lane = threadIdx.x & 31;
    const unsigned lanes_below = (1u << lane) - 1u;
    BinGeom g;
    place_sensor(g, p, fp);
    const float x0 = (float)(it.lt % ts.ntx * 16), y0 = (float)((it.lt / ts.ntx) % ts.nty * 16);
    const float z0 = (float)(it.lt / (ts.ntx * ts.nty) * ts.tz);
    for (int r0 = 0; r0 < it.nr; r0 += THREADS) {  // uniform trip count: the ballots below
        const int r = r0 + (int)threadIdx.x;
        unsigned qm = 0;
        if (r < it.nr) {
            uint32_t rid = A.evals[it.e0 + r];
            if (rid >= (uint32_t)A.bt.N) rid = 0;  // defensive: never read past the ray arrays
            const float4 a4 = A.ray_a[rid];
            sa[r] = a4;
            sc[r] = A.ray_c[rid];
            if (regions) {
                const float ir = 1.0f / p.res;  // K3DOM binning segment: sensor -> point
                qm = region_mask(g.ax, g.ay, g.az, a4.x * ir, a4.y * ir, a4.z * ir, x0, y0, z0, ts.tz,
                                 sd.bin_R + 0.25f);
            }
        }
        if (regions) {
#pragma unroll
            for (int q = 0; q < kRegions; ++q) {
                const unsigned b = __ballot_sync(0xffffffffu, (qm >> q) & 1u);
                if (!b) continue;
                int base = 0;
                if (lane == 0) base = atomicAdd(&rcnt[q], __popc(b));
                base = __shfl_sync(0xffffffffu, base, 0);
                if ((qm >> q) & 1u) reg[q * A.chunk + base + __popc(b & lanes_below)] = (uint16_t)r;
            }
        }
    }
}

// Region of sub-block sb in a 16x16 tile (4x4 sub-blocks per layer).
__device__ __forceinline__ int sb_region(const TileShape& ts, int sb) {
    return ((sb % ts.nsbx) >> 1) + 2 * (((sb / ts.nsbx) % ts.nsby) >> 1);
}

// Pair geometry. For the anchor o of a sub-block and a ray m (FP64, once per lane-ray):
//   par0 = o.u, perp0 = o - par0 u, occ0 = o - m, and par0 - margin, par0 - d_m.
// For a cell c = o + delta (delta small and exact), with dpar = delta.u:
//   projection d_proj = par0 + dpar; perpendicular offset perp0 + delta - dpar u;
//   distance to the free segment [0, margin u] (the three branches of mass_update.cu:57-65)
//   = |perp|^2 + (min(d_proj, 0) + max(d_proj - margin, 0))^2, valid while d_proj < d_m;
//   distance to the point = |occ0 + delta|.
// Every FP32 quantity is O(ls), so the FP32 evaluation keeps ~1e-7 relative accuracy at any
// distance from the sensor (the direct |c|^2 - d_proj^2 form of :60 loses ~1e-5 at 20 m).
//
// stage_pair culls the pair on the sub-block and, for a pair that passes, forms three float4:
// st[0] = (perp0, par0), st[1] = (u, par0 - margin), st[2] = (occ0, par0 - d_m).
//
// The cull bounds the distance from a convex set K (the segment [0, d_m u], or the point) to the
// sub-block's cell centres x = c + h, |h_i| <= e_i, e = (1.5, 1.5, 0.5) res around the centroid c.
// dist(K, .) is convex with gradient D / |D| at c (D = c minus the closest point of K), so
// dist(K, x) >= |D| - (e . |D|) / |D| for every cell centre, where |D| is taken componentwise in
// e . |D|. No cell is within rls = ls (1 + 1e-4) + 1e-3 res of K unless |D|^2 - e . |D| < rls |D|
// (box_reaches). This is tighter than a sphere around c for the flat 4x4x2 sub-block, above all
// for the near-horizontal rays of a LiDAR scan.
//
// *near: the point's sphere of radius ls can reach a cell of the sub-block. For the other rays no
// cell of the sub-block with d_proj >= d_m is within ls of the free segment either (margin <= d_m,
// so such a cell is at least as far from the segment's end as from the point, and the bound above
// keeps 1e-4 ls + 1e-3 res of slack), so their free term needs no d_m test.
__device__ __forceinline__ bool box_reaches(float Dx, float Dy, float Dz, float D2, float hres, float rls2) {
    const float s = fmaf(3.0f * hres, fabsf(Dx) + fabsf(Dy), hres * fabsf(Dz));
    const float t = D2 - s;
    return t < 0.0f || t * t < rls2 * D2;
}

__device__ __forceinline__ bool stage_pair(const float4& a, const double4& cd, double ox, double oy, double oz,
                                           float hres, float rls2, float4 st[3], bool* near) {
    const double par0 = (ox * a.x + oy * a.y + oz * a.z) * cd.z;
    const double sc = par0 * cd.z;
    const double px = ox - sc * a.x, py = oy - sc * a.y, pz = oz - sc * a.z;
    const float ux = (float)(a.x * cd.z), uy = (float)(a.y * cd.z), uz = (float)(a.z * cd.z);
    // centroid = anchor - res/2 on each axis; its perpendicular offset q and its distance qal
    // along the ray beyond [0, d_m], in FP32
    const float qd = -hres * (ux + uy + uz);
    const float qpar = (float)par0 + qd;
    const float qx = (float)px - hres - qd * ux, qy = (float)py - hres - qd * uy, qz = (float)pz - hres - qd * uz;
    const float qal = fminf(qpar, 0.0f) + fmaxf(qpar - a.w, 0.0f);
    const bool hit = box_reaches(fmaf(qal, ux, qx), fmaf(qal, uy, qy), fmaf(qal, uz, qz),
                                 qx * qx + qy * qy + qz * qz + qal * qal, hres, rls2);
    *near = false;
    if (hit) {
        const float ex = (float)(ox - a.x), ey = (float)(oy - a.y), ez = (float)(oz - a.z);
        const float cx = ex - hres, cy = ey - hres, cz = ez - hres;
        st[0] = make_float4((float)px, (float)py, (float)pz, (float)par0);
        st[1] = make_float4(ux, uy, uz, (float)(par0 - cd.y));
        st[2] = make_float4(ex, ey, ez, (float)(par0 - cd.x));
        *near = box_reaches(cx, cy, cz, cx * cx + cy * cy + cz * cz, hres, rls2);
    }
    return hit;
}

// Two FP32 values in one 8-byte register pair for the packed f32x2 instructions of sm_100a: one
// instruction applies the same IEEE operation (round to nearest unless stated) to both halves, so
// each half equals the scalar operation on it.
struct F2 {
    unsigned long long v;
    static __device__ __forceinline__ F2 of(float a, float b) {
        F2 r;
        asm("mov.b64 %0, {%1, %2};" : "=l"(r.v) : "f"(a), "f"(b));
        return r;
    }
    __device__ __forceinline__ void split(float& a, float& b) const {
        asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
    }
};
__device__ __forceinline__ F2 add2(F2 a, F2 b) {
    F2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
    return d;
}
__device__ __forceinline__ F2 add2_rd(F2 a, F2 b) {  // rounded toward -infinity
    F2 d;
    asm("add.rm.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
    return d;
}
__device__ __forceinline__ F2 sub2(F2 a, F2 b) {
    F2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
    return d;
}
__device__ __forceinline__ F2 mul2(F2 a, F2 b) {
    F2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d.v) : "l"(a.v), "l"(b.v));
    return d;
}
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) {
    F2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d.v) : "l"(a.v), "l"(b.v), "l"(c.v));
    return d;
}

// Squared distances from the cell at offset (dx, dy, dz) from the anchor to the free segments
// [0, margin u] of the two rays of a pair record (float4 0-3); *dpar = delta.u for each:
// dp = delta.u, q = p + delta - dp u, al = min(par0 + dp, 0) + max(par0 - margin + dp, 0),
// d^2 = |q|^2 + al^2.
__device__ __forceinline__ F2 free_d2x2(const float4& b0, const float4& b1, const float4& b2, const float4& b3,
                                        F2 DX, F2 DY, F2 DZ, F2* dpar) {
    const F2 ux = F2::of(b2.x, b2.y), uy = F2::of(b2.z, b2.w), uz = F2::of(b3.x, b3.y);
    const F2 dp = fma2(DZ, uz, fma2(DY, uy, mul2(DX, ux)));
    const F2 ndp = mul2(dp, F2::of(-1.0f, -1.0f));  // exact
    const F2 qx = fma2(ndp, ux, add2(F2::of(b0.x, b0.y), DX));
    const F2 qy = fma2(ndp, uy, add2(F2::of(b0.z, b0.w), DY));
    const F2 qz = fma2(ndp, uz, add2(F2::of(b1.x, b1.y), DZ));
    float a0, a1, e0, e1;
    add2(F2::of(b1.z, b1.w), dp).split(a0, a1);  // d_proj
    add2(F2::of(b3.z, b3.w), dp).split(e0, e1);  // d_proj - margin
    const F2 al = add2(F2::of(fminf(a0, 0.0f), fminf(a1, 0.0f)), F2::of(fmaxf(e0, 0.0f), fmaxf(e1, 0.0f)));
    *dpar = dp;
    return fma2(al, al, fma2(qz, qz, fma2(qy, qy, mul2(qx, qx))));
}

// tab_pos for two squared distances: t = d^2 * tscale, then the floor without conversions.
struct TabPos2 {
    TabPos a, b;
};
__device__ __forceinline__ TabPos2 tab_pos2(F2 d2, F2 tscale) {
    const F2 c23 = F2::of(8388608.0f, 8388608.0f);
    const F2 t = mul2(d2, tscale);
    const F2 tr = add2_rd(t, c23);
    const F2 f = sub2(t, sub2(tr, c23));
    float ra, rb;
    tr.split(ra, rb);
    TabPos2 q;
    q.a.i = __float_as_int(ra) - 0x4B000000;
    q.b.i = __float_as_int(rb) - 0x4B000000;
    f.split(q.a.f, q.b.f);
    return q;
}

// Writes the three staged float4 of a passing ray into half (slot & 1) of pair record slot / 2.
__device__ __forceinline__ void stage_put(float* stg, int slot, const float4 st[3]) {
    float* d = stg + (slot >> 1) * kStagePairFloats + (slot & 1);
    d[0] = st[0].x; d[2] = st[0].y; d[4] = st[0].z; d[6] = st[0].w;
    d[8] = st[1].x; d[10] = st[1].y; d[12] = st[1].z; d[14] = st[1].w;
    d[16] = st[2].x; d[18] = st[2].y; d[20] = st[2].z; d[22] = st[2].w;
}

// A pad ray in slot (odd, < 32): perpendicular and point offsets of 1e15 put every cell at a
// squared distance near 3e30 (finite in FP32, far beyond ls^2), and d_proj - d_m = d_proj = 0
// fails the d_proj < d_m test, so the pad adds nothing.
__device__ __forceinline__ void stage_pad(float* stg, int slot) {
    const float4 big = make_float4(1e15f, 1e15f, 1e15f, 0.0f);
    const float4 st[3] = {big, make_float4(0.0f, 0.0f, 0.0f, 0.0f), big};
    stage_put(stg, slot, st);
}

template <int MINB, int THREADS = kEvThreads, bool REGIONS = false>
__global__ void __launch_bounds__(THREADS, MINB) k_bgki(EvArgs A) {
    extern __shared__ __align__(32) unsigned char smem_raw[];
    const BgkiSmem S = bgki_smem(smem_raw, A.chunk, THREADS / 32);
    __shared__ uint32_t s_item;
    __shared__ int s_next_sb, s_last;
    __shared__ SbOrder s_order;
    __shared__ int s_rcnt[kRegions];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned lanes_below = (1u << lane) - 1u;
    const Batch& bt = A.bt;
    const uint32_t total_items = A.item_off[bt.T];
    unsigned nev = 0;      // in-support evaluations of this lane (the roofline's work count)

    for (;;) {
        if (threadIdx.x == 0) {
            s_item = atomicAdd(&A.status->work_counter, 1u);
            s_next_sb = 0;
        }
        if (REGIONS && threadIdx.x < kRegions) s_rcnt[threadIdx.x] = 0;
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= total_items) break;
        const Item it = item_of(bt, A.item_off, A.tile_start, item, A.chunk);
        const SceneDev& sd = bt.sc[it.sc];
        const DevParams& p = sd.p;
        const TileShape ts = sd.ts;
        const FrameParams fp = bt.fp[it.sc];
        const int coff = bt.off->cell[it.sc];
        const float ls2 = p.ls * p.ls;
        const float tscale = (1.0f / ls2) * (float)kKernelTab;  // d^2 -> table position
        const float hres = 0.5f * p.res;
        const float cull_ls2 = sd.cull_ls2;
        const int nsb = ts.nsbx * ts.nsby * (ts.tz / 2);
        const int tbase = it.sc * kKernelTabEntries;  // the scene's table in the texture
        const bool regions = REGIONS && ts.tx == 16 && ts.ty == 16;
        stage_item_rays<THREADS>(A, it, sd, fp, regions, S.a, S.c, S.reg, s_rcnt);
        sb_order_keys(s_order, p, ts, it.lt, nsb, fp.sensor_x, fp.sensor_y, fp.sensor_z);
        __syncthreads();
        sb_order_rank(s_order, nsb);
        __syncthreads();
        const int nr = it.nr;
        for (;;) {
            int sb = 0;
            if (lane == 0) sb = atomicAdd(&s_next_sb, 1);
            sb = __shfl_sync(0xffffffffu, sb, 0);
            if (sb >= nsb) break;
            sb = sb_at(s_order, sb, nsb);
            const CellLoc L = locate(p, ts, it.lt, sb, lane, fp.sensor_x, fp.sensor_y, fp.sensor_z);
            const float dx = L.x - L.ox, dy = L.y - L.oy, dz = L.z - L.oz;  // exact (nearby floats)
            const float ls2c = L.c >= 0 ? ls2 : -1.0f;  // cells outside the grid take no evidence
            const double ox = L.ox, oy = L.oy, oz = L.oz;
            const F2 DX = F2::of(dx, dx), DY = F2::of(dy, dy), DZ = F2::of(dz, dz), TS = F2::of(tscale, tscale);
            float* stg = S.stage + wid * kStageWarpFloats;
            // sums of kernel values rounded to integer units; the unsigned conversion saturates a
            // negative table value (the kernel's max(0, .)) to 0
            unsigned long long ao = 0, af = 0;
            // the rays to cull: the sub-block's region list, or every ray of the item
            const int q = sb_region(ts, sb);
            const int nlist = regions ? s_rcnt[q] : nr;
            const uint16_t* list = S.reg + q * A.chunk;
            for (int g0 = 0; g0 < nlist; g0 += 32) {
                const int j = g0 + lane;
                bool hit = false, near = false;
                float4 st[3];
                if (j < nlist) {
                    const int r = regions ? (int)list[j] : j;
                    hit = stage_pair(S.a[r], S.c[r], ox, oy, oz, hres, cull_ls2, st, &near);
                }
                // compact the passing rays into the warp's staging list, near rays first, two rays
                // to a pair record; an odd count ends in a pad ray that reaches no cell
                const unsigned mnear = __ballot_sync(0xffffffffu, near);
                const unsigned mfar = __ballot_sync(0xffffffffu, hit && !near);
                const int nn = __popc(mnear), nh = nn + __popc(mfar);
                if (hit) stage_put(stg, near ? __popc(mnear & lanes_below) : nn + __popc(mfar & lanes_below), st);
                if ((nh & 1) && lane == 0) stage_pad(stg, nh);
                __syncwarp();
                // pairs holding a ray whose point's sphere can reach the sub-block: occupied
                // (mass_update.cu:48-52) and free (:54-71) evidence; a far ray sharing such a pair
                // adds nothing through the occupied term or the d_proj < d_m test (see stage_pair)
                const int npn = (nn + 1) >> 1, npa = (nh + 1) >> 1;
                for (int k = 0; k < npn; ++k) {
                    const float4* B = reinterpret_cast<const float4*>(stg + k * kStagePairFloats);
                    {  // occupied term
                        const float4 b4 = B[4], b5 = B[5];
                        const F2 vx = add2(F2::of(b4.x, b4.y), DX), vy = add2(F2::of(b4.z, b4.w), DY);
                        const F2 vz = add2(F2::of(b5.x, b5.y), DZ);
                        const F2 d2o = fma2(vz, vz, fma2(vy, vy, mul2(vx, vx)));
                        float oa, ob;
                        d2o.split(oa, ob);
                        const TabPos2 po = tab_pos2(d2o, TS);
                        if (oa < ls2c) { ao += __float2ull_rn(tab_eval_tex(A.ktex, tbase, po.a)); ++nev; }
                        if (ob < ls2c) { ao += __float2ull_rn(tab_eval_tex(A.ktex, tbase, po.b)); ++nev; }
                    }
                    F2 dp;
                    const F2 d2f = free_d2x2(B[0], B[1], B[2], B[3], DX, DY, DZ, &dp);
                    const float4 b5 = B[5];
                    const F2 toend = add2(F2::of(b5.z, b5.w), dp);  // d_proj - d_m
                    float fa, fb, ea, eb;
                    d2f.split(fa, fb);
                    toend.split(ea, eb);
                    const TabPos2 pf = tab_pos2(d2f, TS);
                    if (ea < 0.0f && fa < ls2c) { af += __float2ull_rn(tab_eval_tex(A.ktex, tbase, pf.a)); ++nev; }
                    if (eb < 0.0f && fb < ls2c) { af += __float2ull_rn(tab_eval_tex(A.ktex, tbase, pf.b)); ++nev; }
                }
                // the other pairs: free evidence only
                for (int k = npn; k < npa; ++k) {
                    const float4* B = reinterpret_cast<const float4*>(stg + k * kStagePairFloats);
                    F2 dp;
                    const F2 d2f = free_d2x2(B[0], B[1], B[2], B[3], DX, DY, DZ, &dp);
                    float fa, fb;
                    d2f.split(fa, fb);
                    const TabPos2 pf = tab_pos2(d2f, TS);
                    if (fa < ls2c) { af += __float2ull_rn(tab_eval_tex(A.ktex, tbase, pf.a)); ++nev; }
                    if (fb < ls2c) { af += __float2ull_rn(tab_eval_tex(A.ktex, tbase, pf.b)); ++nev; }
                }
                __syncwarp();
            }
            if (L.c >= 0) {
                unsigned long long* ac = A.acc + 2 * (long)(coff + L.c);
                if (ao) atomicAdd(ac, ao);
                if (af) atomicAdd(ac + 1, af);
            }
        }
        if (!A.fuse_update) {  // the cells are updated by k_k3dom_update_cells after this kernel
            __syncthreads();
            continue;
        }
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) s_last = (atomicAdd(&A.tile_done[it.t], 1u) == it.n_items - 1) ? 1 : 0;
        __syncthreads();
        if (s_last) {
            __threadfence();
            const int tx = it.lt % ts.ntx, ty = (it.lt / ts.ntx) % ts.nty, tz = it.lt / (ts.ntx * ts.nty);
            const int tile_cells = ts.tx * ts.ty * ts.tz;
            for (int li = threadIdx.x; li < tile_cells; li += THREADS) {
                const int lx = li % ts.tx, ly = (li / ts.tx) % ts.ty, lz = li / (ts.tx * ts.ty);
                const int ix = tx * ts.tx + lx, iy = ty * ts.ty + ly, iz = tz * ts.tz + lz;
                if (ix >= p.G || iy >= p.G || iz >= p.Gz) continue;
                const int c = coff + ix + p.G * iy + p.G * p.G * iz;
                // every chunk of the tile has added its share (fence + tile counter above); read
                // the totals from L2 and clear only what was written
                unsigned long long* ac = A.acc + 2 * (long)c;
                const long long fo = (long long)__ldcg(ac);
                const long long ff = (long long)__ldcg(ac + 1);
                if (fo) __stcg(ac, 0ull);
                if (ff) __stcg(ac + 1, 0ull);
                k3dom_cell_update(p, fp.gamma_dt, c, (double)fo * sd.fx_inv, (double)ff * sd.fx_inv, A.cs, A.cw,
                                  A.first_frame != 0);
            }
            if (threadIdx.x == 0) A.tile_done[it.t] = 0;
        }
        __syncthreads();
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nev += __shfl_xor_sync(0xffffffffu, nev, o);
    if (lane == 0 && nev) atomicAdd(&A.status->kernel_evals, (unsigned long long)nev);
}

// ================================================================ DS-PHD/MIB
struct DsMeas {
    float occ, free_m;
};

// The measurement masses of measurement_grid.cu:98-157 from the neighbour summary.
__device__ __forceinline__ DsMeas ds_meas_from(const DevParams& p, float acs, int nb, bool all_farther,
                                               float max_occ) {
    DsMeas m;
    if (nb == 0) {
        m.occ = 0.0f;
        m.free_m = 0.0f;
        return m;
    }
    float mo, mf;
    if (all_farther) {
        // pFree (:41-50): p_min + r / max_range * (p_max - p_min)
        const float r = sqrtf(acs);
        const float unc = __fadd_rn(0.15f, __fmul_rn(__fdiv_rn(r, p.max_range), __fsub_rn(1.0f, 0.15f)));
        if (max_occ > unc) {
            mo = max_occ;
            mf = 0.0f;
        } else {
            mo = 0.0f;
            mf = __fsub_rn(1.0f, unc);
        }
    } else {
        mo = max_occ > 0.5f ? max_occ : 0.0f;
        mf = 0.0f;
    }
    const float eps = 0.00001f;
    m.occ = fmaxf(eps, fminf(__fsub_rn(1.0f, eps), mo));
    m.free_m = fmaxf(eps, fminf(__fsub_rn(1.0f, eps), mf));
    return m;
}

// update_masses (src/dsphdmib/kernel/mass_update.cu:17-30) keeping its double promotions.
__device__ __forceinline__ void ds_update_masses(float mop, float mfp, DsMeas mc, float* occ, float* fr) {
    const float unknown_pred = (float)(1.0 - (double)mop - (double)mfp);
    const float meas_unknown = (float)(1.0 - (double)mc.free_m - (double)mc.occ);
    const float K = __fadd_rn(__fmul_rn(mfp, mc.occ), __fmul_rn(mop, mc.free_m));
    const float no = __fadd_rn(__fadd_rn(__fmul_rn(mop, meas_unknown), __fmul_rn(unknown_pred, mc.occ)),
                               __fmul_rn(mop, mc.occ));
    const float nf = __fadd_rn(__fadd_rn(__fmul_rn(mfp, meas_unknown), __fmul_rn(unknown_pred, mc.free_m)),
                               __fmul_rn(mfp, mc.free_m));
    const double den = 1.0 - (double)K;
    *occ = (float)((double)no / den);
    *fr = (float)((double)nf / den);
}

__device__ void ds_cell_update(const DevParams& p, int c, DsMeas mc, CellState cs, CellWork cw, bool first_frame) {
    cw.meas_occ[c] = mc.occ;
    cw.meas_free[c] = mc.free_m;
    if (first_frame) {
        cs.born_m[c] = mc.occ;  // copyMassesKernel (measurement_grid.cu:55-62)
        return;
    }
    const int start = cw.start[c];
    const bool has = start >= 0;
    const float free0 = cs.free_m[c];
    float occ_up, free_up, rho_b = 0.0f, mop = 0.0f, divisor = 0.0f;
    if (has) {
        mop = cw.sum_w[c];
        if (mop > 1.0f) {
            divisor = mop;  // normalize_weights (:37-44), applied in the reweight kernel
            mop = 1.0f;
        }
        const float mfp = fminf(__fmul_rn(0.9f, free0), __fsub_rn(1.0f, mop));
        ds_update_masses(mop, mfp, mc, &occ_up, &free_up);
        // separate_newborn_part (:32-35) with its double promotions
        const double om = 1.0 - (double)mop;
        rho_b = (float)(((double)__fmul_rn(occ_up, p.p_B) * om) / ((double)mop + (double)p.p_B * om));
    } else {
        const float m_occ = cs.occ_m[c];
        const float m_free = fminf(__fmul_rn(0.9f, free0), __fsub_rn(1.0f, m_occ));
        ds_update_masses(m_occ, m_free, mc, &occ_up, &free_up);
    }
    const float pers = __fsub_rn(occ_up, rho_b);
    cs.born_m[c] = rho_b;
    cs.pers_m[c] = pers;
    cs.free_m[c] = free_up;
    cs.occ_m[c] = occ_up;
    cs.pred_m[c] = mop;
    const float mu_UA = has ? calc_norm(mop, pers) : 0.0f;
    cw.factor[c] = mu_UA;
    cw.divisor[c] = divisor;
    float vx = 0.0f, vy = 0.0f, vz = 0.0f;
    if (has && pers > 0.0f) {
        float sx = cw.sum_wvx[c], sy = cw.sum_wvy[c], sz = cw.sum_wvz[c];
        if (divisor > 0.0f) {
            sx /= divisor;
            sy /= divisor;
            sz /= divisor;
        }
        vx = (mu_UA * sx) / pers;
        vy = (mu_UA * sy) / pers;
        vz = (mu_UA * sz) / pers;
    }
    cs.mvx[c] = vx;
    cs.mvy[c] = vy;
    cs.mvz[c] = vz;
}

// Neighbour test of measurement_grid.cu:88-99 in the reference's FP32 operation order.
__device__ __forceinline__ bool ds_is_neighbor(float x, float y, float z, float acs, float4 m, float wr2) {
    const float ip = __fadd_rn(__fadd_rn(__fmul_rn(x, m.x), __fmul_rn(y, m.y)), __fmul_rn(z, m.z));
    return ip > 0.0f && __fsub_rn(acs, __fdiv_rn(__fmul_rn(ip, ip), m.w)) < wr2;
}

// pOcc (measurement_grid.cu:28-39)
__device__ __forceinline__ float ds_pocc(float x, float y, float z, float4 m, float delta) {
    const float dx = __fsub_rn(x, m.x), dy = __fsub_rn(y, m.y), dz = __fsub_rn(z, m.z);
    const float r_sqr = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
    const float delta_sqr = __fmul_rn(delta, delta);
    return __fmul_rn(0.95f, expf(__fdiv_rn(__fmul_rn(-0.5f, r_sqr), delta_sqr)));
}

// Pass COUNT (multi-chunk tiles, every chunk but the last): per (item, cell) number of
// neighbours. Pass !COUNT: each cell takes its first (100 - neighbours in earlier chunks)
// neighbours of the chunk, in list order, so the kept set is the reference's first 100 rays in
// input order (measurement_grid.cu:86-97). Per-chunk summaries (any neighbour, all farther,
// largest pOcc) are combined per cell with integer atomics; the last CTA of a tile runs the
// measurement-to-mass step for the whole tile.
constexpr int kMaxTileCells = 16 * 16 * 8;

template <bool COUNT>
__global__ void __launch_bounds__(kEvThreads, COUNT ? 5 : 4) k_dsgrid(EvArgs A) {
    __shared__ float4 sa[kChunk];  // (m, |m|^2)
    __shared__ float4 su[kChunk];  // (m / |m|, 0)
    __shared__ uint16_t s_cand[kEvWarps][32];
    __shared__ uint16_t s_reg[kRegions][kChunk];  // region lists, in input order
    __shared__ int s_wq[2][kEvWarps][kRegions];     // per-warp region counts of a staging step
    __shared__ int s_rcnt[kRegions];
    __shared__ uint32_t s_item;
    __shared__ int s_next_sb, s_last;
    __shared__ SbOrder s_order;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned lanes_below = (1u << lane) - 1u;
    const Batch& bt = A.bt;
    const uint32_t total_items = A.item_off[bt.T];
    unsigned int* counter = COUNT ? &A.status->work_counter2 : &A.status->work_counter;
    uint32_t* part_max = reinterpret_cast<uint32_t*>(A.acc);
    uint32_t* part_flags = part_max + bt.C;
    unsigned nev = 0;  // accepted neighbours of this lane (the roofline's work count, final pass)

    for (;;) {
        if (threadIdx.x == 0) {
            s_item = atomicAdd(counter, 1u);
            s_next_sb = 0;
        }
        if (threadIdx.x < kRegions) s_rcnt[threadIdx.x] = 0;
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= total_items) break;
        const Item it = item_of(bt, A.item_off, A.tile_start, item, A.chunk);
        if (COUNT && (it.n_items == 1 || it.k == it.n_items - 1)) {  // uniform across the block
            __syncthreads();
            continue;
        }
        const SceneDev& sd = bt.sc[it.sc];
        const DevParams& p = sd.p;
        const TileShape ts = sd.ts;
        const FrameParams fp = bt.fp[it.sc];
        const int coff = bt.off->cell[it.sc];
        const int nsb = ts.nsbx * ts.nsby * (ts.tz / 2);
        const float hres = 0.5f * p.res;
        // Rays staged with their unit directions; in a 16x16 tile each is also listed, in input
        // order, under the 8x8-cell columns its binned half-line (sensor -> grid exit along m)
        // meets within the binning radius, so a sub-block visits only its column's rays, still in
        // input order (the first-100 rule).
        const bool regions = ts.tx == 16 && ts.ty == 16;
        BinGeom g;
        place_sensor(g, p, fp);
        const float x0 = (float)(it.lt % ts.ntx * 16), y0 = (float)((it.lt / ts.ntx) % ts.nty * 16);
        const float z0 = (float)(it.lt / (ts.ntx * ts.nty) * ts.tz);
        const float Lc = sqrtf((float)(2 * p.G * p.G + p.Gz * p.Gz)) + 2.0f * sd.bin_R + 4.0f;  // cells
        int step = 0;
        for (int r0 = 0; r0 < it.nr; r0 += kEvThreads, ++step) {  // uniform trip count
            const int r = r0 + (int)threadIdx.x;
            unsigned qm = 0;
            if (r < it.nr) {
                uint32_t rid = A.evals[it.e0 + r];
                if (rid >= (uint32_t)bt.N) rid = 0;
                const float4 a = A.ray_a[rid];
                sa[r] = a;
                const float len = sqrtf(a.w);
                const float inv = len > 0.0f ? 1.0f / len : 0.0f;
                const float4 u = make_float4(a.x * inv, a.y * inv, a.z * inv, 0.0f);
                su[r] = u;
                if (regions)
                    qm = region_mask(g.ax, g.ay, g.az, u.x * Lc, u.y * Lc, u.z * Lc, x0, y0, z0, ts.tz,
                                     sd.bin_R + 0.25f);
            }
            if (regions) {
                unsigned b[kRegions];
#pragma unroll
                for (int q = 0; q < kRegions; ++q) b[q] = __ballot_sync(0xffffffffu, (qm >> q) & 1u);
                int(*wq)[kRegions] = s_wq[step & 1];
                if (lane == 0) {
#pragma unroll
                    for (int q = 0; q < kRegions; ++q) wq[wid][q] = __popc(b[q]);
                }
                __syncthreads();
#pragma unroll
                for (int q = 0; q < kRegions; ++q) {
                    if (!((qm >> q) & 1u)) continue;
                    int pos = s_rcnt[q] + __popc(b[q] & lanes_below);
                    for (int w = 0; w < wid; ++w) pos += wq[w][q];
                    s_reg[q][pos] = (uint16_t)r;
                }
                __syncthreads();
                if (threadIdx.x < kRegions) {
                    int t = 0;
                    for (int w = 0; w < kEvWarps; ++w) t += wq[w][threadIdx.x];
                    s_rcnt[threadIdx.x] += t;
                }
            }
        }
        sb_order_keys(s_order, p, ts, it.lt, nsb, fp.sensor_x, fp.sensor_y, fp.sensor_z);
        __syncthreads();
        sb_order_rank(s_order, nsb);
        __syncthreads();
        const int nr = it.nr;
        for (;;) {
            int sb = 0;
            if (lane == 0) sb = atomicAdd(&s_next_sb, 1);
            sb = __shfl_sync(0xffffffffu, sb, 0);
            if (sb >= nsb) break;
            sb = sb_at(s_order, sb, nsb);
            const CellLoc L = locate(p, ts, it.lt, sb, lane, fp.sensor_x, fp.sensor_y, fp.sensor_z);
            const float acs = __fadd_rn(__fadd_rn(__fmul_rn(L.x, L.x), __fmul_rn(L.y, L.y)), __fmul_rn(L.z, L.z));
            int quota = kDsMaxNeighbors;
            if (!COUNT && it.n_items > 1) {
                int pre = 0;
                const long base = (long)A.item_off[it.t] * kMaxTileCells;
                for (uint32_t kk = 0; kk < it.k; ++kk) {
                    const long idx = base + (long)kk * kMaxTileCells + L.local;
                    pre += (idx < A.ds_count_capacity) ? (int)A.ds_counts[idx] : 0;
                }
                quota = max(0, kDsMaxNeighbors - pre);
            }
            if (L.c < 0) quota = 0;
            int nb = 0;
            bool all_far = true;
            float mx = 0.0f;
            const int q = sb_region(ts, sb);
            const int nlist = regions ? s_rcnt[q] : nr;
            if (__any_sync(0xffffffffu, quota > 0)) {
                for (int g0 = 0; g0 < nlist; g0 += 32) {
                    const int jl = g0 + lane;
                    const int r = regions ? (jl < nlist ? (int)s_reg[q][jl] : 0) : jl;
                    bool hit = false;
                    if (jl < nlist) {
                        // box bound on the distance from the half-line through m to the sub-block's
                        // cell centres (the K3DOM cull's bound, with the window as the radius)
                        const float4 u = su[r];
                        const float qx = L.ox - hres, qy = L.oy - hres, qz = L.oz - hres;
                        const float tproj = fmaxf(qx * u.x + qy * u.y + qz * u.z, 0.0f);
                        const float Dx = qx - tproj * u.x, Dy = qy - tproj * u.y, Dz = qz - tproj * u.z;
                        hit = box_reaches(Dx, Dy, Dz, Dx * Dx + Dy * Dy + Dz * Dz, hres, sd.cull_ls2);
                    }
                    // candidates in input order (the first-100 rule counts them in that order)
                    const unsigned mask = __ballot_sync(0xffffffffu, hit);
                    if (hit) s_cand[wid][__popc(mask & lanes_below)] = (uint16_t)r;
                    __syncwarp();
                    const int ncand = __popc(mask);
                    for (int k = 0; k < ncand; ++k) {
                        const float4 a = sa[s_cand[wid][k]];
                        if (nb < quota && ds_is_neighbor(L.x, L.y, L.z, acs, a, sd.wr2)) {
                            ++nb;
                            if (!COUNT) {
                                ++nev;
                                if (acs > a.w) all_far = false;
                                const float o = ds_pocc(L.x, L.y, L.z, a, p.meas_occ_stddev);
                                if (o > mx) mx = o;
                            }
                        }
                    }
                    __syncwarp();
                    if (!__any_sync(0xffffffffu, nb < quota)) break;
                }
            }
            if (COUNT) {
                if (L.c >= 0) {
                    const long idx = (long)item * kMaxTileCells + L.local;
                    if (idx < A.ds_count_capacity) A.ds_counts[idx] = (uint8_t)nb;
                }
            } else if (L.c >= 0 && nb > 0) {
                const int c = coff + L.c;
                atomicMax(&part_max[c], __float_as_uint(mx));
                atomicOr(&part_flags[c], 1u | (all_far ? 0u : 2u));
            }
        }
        if (COUNT) {
            __syncthreads();
            continue;
        }
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) s_last = (atomicAdd(&A.tile_done[it.t], 1u) == it.n_items - 1) ? 1 : 0;
        __syncthreads();
        if (s_last) {
            __threadfence();
            const int tx = it.lt % ts.ntx, ty = (it.lt / ts.ntx) % ts.nty, tz = it.lt / (ts.ntx * ts.nty);
            const int tile_cells = ts.tx * ts.ty * ts.tz;
            for (int li = threadIdx.x; li < tile_cells; li += kEvThreads) {
                const int lx = li % ts.tx, ly = (li / ts.tx) % ts.ty, lz = li / (ts.tx * ts.ty);
                const int ix = tx * ts.tx + lx, iy = ty * ts.ty + ly, iz = tz * ts.tz + lz;
                if (ix >= p.G || iy >= p.G || iz >= p.Gz) continue;
                const int c = coff + ix + p.G * iy + p.G * p.G * iz;
                const uint32_t m = __ldcg(&part_max[c]);
                const uint32_t f = __ldcg(&part_flags[c]);
                if (m) __stcg(&part_max[c], 0u);
                if (f) __stcg(&part_flags[c], 0u);
                float x, y, z;
                centre_xyz(ix, iy, iz, p, fp.sensor_x, fp.sensor_y, fp.sensor_z, &x, &y, &z);
                const float acs = __fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z));
                const DsMeas mc = ds_meas_from(p, acs, (f & 1u) ? 1 : 0, (f & 2u) == 0, __uint_as_float(m));
                ds_cell_update(p, c, mc, A.cs, A.cw, A.first_frame != 0);
            }
            if (threadIdx.x == 0) A.tile_done[it.t] = 0;
        }
        __syncthreads();
    }
    if (!COUNT) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) nev += __shfl_xor_sync(0xffffffffu, nev, o);
        if (lane == 0 && nev) atomicAdd(&A.status->kernel_evals, (unsigned long long)nev);
    }
}

// ================================================================ launchers
static EvArgs make_args(const Batch& bt, RayBuffers& rb, CellState cs, CellWork cw, bool first_frame,
                        DevStatus* status) {
    EvArgs A;
    A.bt = bt;
    A.item_off = rb.item_off;
    A.tile_start = rb.tile_start;
    A.evals = rb.evals2;
    A.ray_a = rb.ray_a;
    A.ray_c = rb.ray_c;
    A.ktab = rb.ktab;
    A.tile_done = rb.tile_done;
    A.acc = rb.acc;
    A.ds_counts = rb.ds_counts;
    A.ds_count_capacity = rb.ds_count_capacity;
    A.cs = cs;
    A.cw = cw;
    A.status = status;
    A.first_frame = first_frame ? 1 : 0;
    A.chunk = rb.chunk;
    A.fuse_update = 1;
    A.ktex = rb.ktex;
    return A;
}

// ================================================================ calibration sums
// For the differentiable update: per cell and frame, the sums of the unit-amplitude sparse
// kernel f(d/ls) over the occupied and free pairs, and of d f(d/ls) / d ls (times ls, i.e.
// -x f'(x)), from the same tiles, culls and pair geometry as k_bgki. Both are summed exactly
// in fixed point (units of 2^-40), so the loss and its gradient are deterministic. No per-pair
// value is stored: the derivative is formed in the same pass as the value.
//
// f(x) = max(0, (2 + cos 2 pi x)(1 - x) / 3 + sin(2 pi x) / (2 * 3.141592)), mass_update.cu:24-26.
static double unit_kernel(double x) {
    const double v = (2.0 + std::cos(M_PI * 2.0 * x)) * (1.0 - x) / 3.0 + std::sin(M_PI * 2.0 * x) / (2.0 * 3.141592);
    return v > 0.0 ? v : 0.0;
}
// -x f'(x) where f > 0 (0 where the clamp is active)
static double unit_kernel_dls(double x) {
    const double v = (2.0 + std::cos(M_PI * 2.0 * x)) * (1.0 - x) / 3.0 + std::sin(M_PI * 2.0 * x) / (2.0 * 3.141592);
    if (!(v > 0.0)) return 0.0;
    const double fp = (-2.0 * M_PI * std::sin(M_PI * 2.0 * x) * (1.0 - x) - (2.0 + std::cos(M_PI * 2.0 * x))) / 3.0 +
                      2.0 * M_PI * std::cos(M_PI * 2.0 * x) / (2.0 * 3.141592);
    return -x * fp;
}

static void build_table(double (*fn)(double), double scale, float4* out) {
    for (int i = 0; i < kKernelTab; ++i) {
        double y[4];
        for (int j = 0; j < 4; ++j) y[j] = scale * fn(std::sqrt(std::min(1.0, (i + j / 3.0) / kKernelTab)));
        const double c0 = y[0];
        const double c1 = -5.5 * y[0] + 9.0 * y[1] - 4.5 * y[2] + y[3];
        const double c2 = 9.0 * y[0] - 22.5 * y[1] + 18.0 * y[2] - 4.5 * y[3];
        const double c3 = -4.5 * y[0] + 13.5 * y[1] - 13.5 * y[2] + 4.5 * y[3];
        out[i] = make_float4((float)c0, (float)c1, (float)c2, (float)c3);
    }
    out[kKernelTab] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

void build_calib_tables(float4* f_tab, float4* dls_tab) {
    build_table(unit_kernel, std::ldexp(1.0, kCalibShift), f_tab);
    build_table(unit_kernel_dls, std::ldexp(1.0, kCalibShift), dls_tab);
}

// Shared memory of k_bgki_sums (dynamic, sized by the work item's ray count).
struct CalibSmem {
    float4* ftab;            // [kKernelTabEntries] unit kernel f, fixed-point scale folded in
    float4* htab;            // [kKernelTabEntries] -x f'(x), same scale
    float* stage;            // [kEvWarps][kStageWarpFloats] pair records, as in k_bgki
    float4* a;               // [chunk]
    double4* c;              // [chunk]
    uint16_t* reg;           // [kRegions][chunk] (region builds)
};

constexpr size_t kCalibFixedBytes =
    2 * sizeof(float4) * kKernelTabEntries + sizeof(float) * (size_t)kEvWarps * kStageWarpFloats;

inline size_t calib_smem_bytes(int chunk, bool regions = false) {
    return ((kCalibFixedBytes + 31) & ~(size_t)31) + (size_t)chunk * (sizeof(float4) + sizeof(double4)) +
           (regions ? (size_t)kRegions * chunk * sizeof(uint16_t) : 0);
}

__device__ __forceinline__ CalibSmem calib_smem(unsigned char* base, int chunk) {
    CalibSmem S;
    S.ftab = reinterpret_cast<float4*>(base);
    S.htab = S.ftab + kKernelTabEntries;
    S.stage = reinterpret_cast<float*>(base + 2 * sizeof(float4) * kKernelTabEntries);
    const size_t off = (kCalibFixedBytes + 31) & ~(size_t)31;
    S.c = reinterpret_cast<double4*>(base + off);
    S.a = reinterpret_cast<float4*>(base + off + sizeof(double4) * (size_t)chunk);
    S.reg = reinterpret_cast<uint16_t*>(base + off + (sizeof(double4) + sizeof(float4)) * (size_t)chunk);
    return S;
}

// acc4: 4 signed 64-bit sums per cell (f occ, f free, -x f' occ, -x f' free), in units. Same
// tiles, culls and pair geometry as k_bgki; each value is rounded once to an integer number of
// units (round to nearest even).
template <int MINB, bool REGIONS = false>
__global__ void __launch_bounds__(kEvThreads, MINB) k_bgki_sums(EvArgs A, const float4* __restrict__ htab,
                                                               unsigned long long* __restrict__ acc4) {
    extern __shared__ __align__(32) unsigned char smem_raw[];
    const CalibSmem S = calib_smem(smem_raw, A.chunk);
    __shared__ uint32_t s_item;
    __shared__ int s_next_sb;
    __shared__ SbOrder s_order;
    __shared__ int s_rcnt[kRegions];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned lanes_below = (1u << lane) - 1u;
    const Batch& bt = A.bt;
    const uint32_t total_items = A.item_off[bt.T];
    for (int i = threadIdx.x; i < kKernelTabEntries; i += kEvThreads) {
        S.ftab[i] = A.ktab[i];
        S.htab[i] = htab[i];
    }
    for (;;) {
        if (threadIdx.x == 0) {
            s_item = atomicAdd(&A.status->work_counter, 1u);
            s_next_sb = 0;
        }
        if (REGIONS && threadIdx.x < kRegions) s_rcnt[threadIdx.x] = 0;
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= total_items) break;
        const Item it = item_of(bt, A.item_off, A.tile_start, item, A.chunk);
        const SceneDev& sd = bt.sc[it.sc];
        const DevParams& p = sd.p;
        const TileShape ts = sd.ts;
        const FrameParams fp = bt.fp[it.sc];
        const int coff = bt.off->cell[it.sc];
        const float ls2 = p.ls * p.ls;
        const float tscale = (1.0f / ls2) * (float)kKernelTab;  // d^2 -> table position
        const float hres = 0.5f * p.res;
        const float cull_ls2 = sd.cull_ls2;
        const int nsb = ts.nsbx * ts.nsby * (ts.tz / 2);
        const bool regions = REGIONS && ts.tx == 16 && ts.ty == 16;
        stage_item_rays<kEvThreads>(A, it, sd, fp, regions, S.a, S.c, S.reg, s_rcnt);
        sb_order_keys(s_order, p, ts, it.lt, nsb, fp.sensor_x, fp.sensor_y, fp.sensor_z);
        __syncthreads();
        sb_order_rank(s_order, nsb);
        __syncthreads();
        const int nr = it.nr;
        for (;;) {
            int sb = 0;
            if (lane == 0) sb = atomicAdd(&s_next_sb, 1);
            sb = __shfl_sync(0xffffffffu, sb, 0);
            if (sb >= nsb) break;
            sb = sb_at(s_order, sb, nsb);
            const CellLoc L = locate(p, ts, it.lt, sb, lane, fp.sensor_x, fp.sensor_y, fp.sensor_z);
            const float dx = L.x - L.ox, dy = L.y - L.oy, dz = L.z - L.oz;
            const float ls2c = L.c >= 0 ? ls2 : -1.0f;
            const double ox = L.ox, oy = L.oy, oz = L.oz;
            const F2 DX = F2::of(dx, dx), DY = F2::of(dy, dy), DZ = F2::of(dz, dz), TS = F2::of(tscale, tscale);
            float* stg = S.stage + wid * kStageWarpFloats;
            long long fo = 0, ff = 0, ho = 0, hf = 0;
            const int q = sb_region(ts, sb);
            const int nlist = regions ? s_rcnt[q] : nr;
            const uint16_t* list = S.reg + q * A.chunk;
            // one in-support evaluation: f (clamped at 0, as the kernel is) and -x f' at position t
            auto eval = [&](TabPos t, long long& f, long long& h) {
                f += __float2ll_rn(fmaxf(tab_eval(S.ftab, t), 0.0f));
                h += __float2ll_rn(tab_eval(S.htab, t));
            };
            for (int g0 = 0; g0 < nlist; g0 += 32) {
                const int j = g0 + lane;
                bool hit = false, near = false;
                float4 st[3];
                if (j < nlist) {
                    const int r = regions ? (int)list[j] : j;
                    hit = stage_pair(S.a[r], S.c[r], ox, oy, oz, hres, cull_ls2, st, &near);
                }
                // the staging of k_bgki: near rays first, two to a pair record, a pad ray last
                const unsigned mnear = __ballot_sync(0xffffffffu, near);
                const unsigned mfar = __ballot_sync(0xffffffffu, hit && !near);
                const int nn = __popc(mnear), nh = nn + __popc(mfar);
                if (hit) stage_put(stg, near ? __popc(mnear & lanes_below) : nn + __popc(mfar & lanes_below), st);
                if ((nh & 1) && lane == 0) stage_pad(stg, nh);
                __syncwarp();
                const int npn = (nn + 1) >> 1, npa = (nh + 1) >> 1;
                for (int k = 0; k < npn; ++k) {
                    const float4* B = reinterpret_cast<const float4*>(stg + k * kStagePairFloats);
                    {  // occupied term
                        const float4 b4 = B[4], b5 = B[5];
                        const F2 vx = add2(F2::of(b4.x, b4.y), DX), vy = add2(F2::of(b4.z, b4.w), DY);
                        const F2 vz = add2(F2::of(b5.x, b5.y), DZ);
                        const F2 d2o = fma2(vz, vz, fma2(vy, vy, mul2(vx, vx)));
                        float oa, ob;
                        d2o.split(oa, ob);
                        const TabPos2 po = tab_pos2(d2o, TS);
                        if (oa < ls2c) eval(po.a, fo, ho);
                        if (ob < ls2c) eval(po.b, fo, ho);
                    }
                    F2 dp;
                    const F2 d2f = free_d2x2(B[0], B[1], B[2], B[3], DX, DY, DZ, &dp);
                    const float4 b5 = B[5];
                    const F2 toend = add2(F2::of(b5.z, b5.w), dp);  // d_proj - d_m
                    float fa, fb, ea, eb;
                    d2f.split(fa, fb);
                    toend.split(ea, eb);
                    const TabPos2 pf = tab_pos2(d2f, TS);
                    if (ea < 0.0f && fa < ls2c) eval(pf.a, ff, hf);
                    if (eb < 0.0f && fb < ls2c) eval(pf.b, ff, hf);
                }
                for (int k = npn; k < npa; ++k) {
                    const float4* B = reinterpret_cast<const float4*>(stg + k * kStagePairFloats);
                    F2 dp;
                    const F2 d2f = free_d2x2(B[0], B[1], B[2], B[3], DX, DY, DZ, &dp);
                    float fa, fb;
                    d2f.split(fa, fb);
                    const TabPos2 pf = tab_pos2(d2f, TS);
                    if (fa < ls2c) eval(pf.a, ff, hf);
                    if (fb < ls2c) eval(pf.b, ff, hf);
                }
                __syncwarp();
            }
            if (L.c >= 0) {
                unsigned long long* ac = acc4 + 4 * (long)(coff + L.c);
                if (fo) atomicAdd(ac, (unsigned long long)fo);
                if (ff) atomicAdd(ac + 1, (unsigned long long)ff);
                if (ho) atomicAdd(ac + 2, (unsigned long long)ho);
                if (hf) atomicAdd(ac + 3, (unsigned long long)hf);
            }
        }
        __syncthreads();
    }
}

cudaError_t launch_bgki_sums(const Batch& bt, RayBuffers& rb, const float4* f_tab, const float4* dls_tab,
                             unsigned long long* acc4, DevStatus* status, int num_sms, cudaStream_t st) {
    if (rb.chunk < 32 || rb.chunk > kChunk) return cudaErrorInvalidValue;
    EvArgs A = make_args(bt, rb, CellState{}, CellWork{}, false, status);
    A.ktab = f_tab;
    // 4 CTAs per SM with region lists up to kCalibChunk rays per item, else 3 without them
    const bool small = rb.chunk <= kCalibChunk;
    const size_t sm = calib_smem_bytes(rb.chunk, small);
    auto kern = small ? k_bgki_sums<4, true> : k_bgki_sums<3>;
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kEvThreads, sm);
    ++g_launches;
    kern<<<num_sms * std::max(1, per_sm), kEvThreads, sm, st>>>(A, dls_tab, acc4);
    return cudaGetLastError();
}

// The K3DOM evidence launch is persistent: one CTA per resident slot of the build the chunk selects
// (128 threads at <= 256 rays, 256 threads with region lists at <= 512, 256 threads at <= 1024).
struct BgkiLaunch {
    int blocks, threads;
    size_t smem;
};

static BgkiLaunch bgki_launch(int chunk) {
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    BgkiLaunch L;
    if (chunk <= kSmallChunk) {
        L.threads = kSmallWarps * 32;
        L.smem = bgki_smem_bytes(chunk, kSmallWarps);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bgki<8, kSmallWarps * 32>, L.threads, L.smem);
    } else if (chunk <= 512) {
        L.threads = kEvThreads;
        L.smem = bgki_smem_bytes(chunk, kEvWarps, true);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bgki<4, kEvThreads, true>, L.threads, L.smem);
    } else {
        L.threads = kEvThreads;
        L.smem = bgki_smem_bytes(chunk);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bgki<3>, L.threads, L.smem);
    }
    L.blocks = sms * std::max(1, per_sm);
    return L;
}

int k3dom_evidence_blocks(int chunk) { return bgki_launch(chunk).blocks; }

// Work items of up to 512 rays leave shared memory for a fourth CTA per SM; that build is limited
// to 64 registers. Items of up to 256 rays run in 128-thread CTAs, 8 per SM. Both builds compute the same sums (exactly), so the choice is speed only.
cudaError_t launch_k3dom_evidence(const Batch& bt, RayBuffers& rb, CellState cs, CellWork cw, bool first_frame,
                                  DevStatus* status, cudaStream_t st, bool fuse_update) {
    if (rb.chunk < 32 || rb.chunk > kChunk) return cudaErrorInvalidValue;
    EvArgs A = make_args(bt, rb, cs, cw, first_frame, status);
    A.fuse_update = fuse_update ? 1 : 0;
    const BgkiLaunch L = bgki_launch(rb.chunk);
    ++g_launches;
    if (rb.chunk <= kSmallChunk)  // 128-thread CTAs: 8 per SM, each item's end waits on 4 warps
        k_bgki<8, kSmallWarps * 32><<<L.blocks, L.threads, L.smem, st>>>(A);
    else if (rb.chunk <= 512)
        k_bgki<4, kEvThreads, true><<<L.blocks, L.threads, L.smem, st>>>(A);
    else
        k_bgki<3><<<L.blocks, L.threads, L.smem, st>>>(A);
    return cudaGetLastError();
}

// The cell update of k_bgki's tile tails as a pass of its own over every cell: a steady frame
// accumulates the evidence beside prediction and assignment (the evidence needs only the ray
// lists) and updates the cells once the particles' per-cell sums are in. Each cell's two
// fixed-point sums are read and cleared, then k3dom_cell_update runs as in the tail: same inputs,
// same bits.
__global__ void __launch_bounds__(kBlock) k_k3dom_update_cells(EvArgs A) {
    const Batch& bt = A.bt;
    ulonglong2* acc = reinterpret_cast<ulonglong2*>(A.acc);  // (occupied, free) per cell
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < bt.C; c += (long)gridDim.x * blockDim.x) {
        const int sc = scene_of(bt.off->cell, bt.S, (int)c);
        const SceneDev& sd = bt.sc[sc];
        const ulonglong2 v = acc[c];
        if (v.x || v.y) acc[c] = make_ulonglong2(0ull, 0ull);
        k3dom_cell_update(sd.p, bt.fp[sc].gamma_dt, (int)c, (double)(long long)v.x * sd.fx_inv,
                          (double)(long long)v.y * sd.fx_inv, A.cs, A.cw, A.first_frame != 0);
    }
}

// The same pass with each CTA's inputs brought into shared memory by bulk copies: the pass is
// latency bound on its per-cell reads, and one cp.async.bulk per input array (8 arrays of 1,024
// cells and the fixed-point sums, 48 KB per CTA, completed on one mbarrier) puts all of a CTA's
// bytes in flight at once without holding them in registers. Each copy is a plain one-CTA copy of
// this GPU's own memory. Every array base is 16-byte aligned (checked by the
// launcher) and a full tile starts at a multiple of 4 KB, as the copies require; the last, partial
// tile reads its cells directly. The wait is bounded: when it runs out the CTA records
// copy_timeout, waits (bounded again) for its copies to land, and skips its cells.
constexpr int kUcCells = 1024;
constexpr int kUcThreads = 256;
constexpr uint32_t kUcMaxPolls = 1u << 22;
constexpr size_t kUcSmem = 8 * sizeof(float) * kUcCells + sizeof(ulonglong2) * kUcCells;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :
                 : "r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// Polls the barrier's phase 0 at most max_polls times; true once it has completed.
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t max_polls) {
    for (uint32_t it = 0; it < max_polls; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_addr(bar))
            : "memory");
        if (done) return true;
    }
    return false;
}

__global__ void __launch_bounds__(kUcThreads) k_k3dom_update_cells_bulk(EvArgs A) {
    extern __shared__ __align__(16) unsigned char uc_smem[];
    __shared__ __align__(8) uint64_t bar;
    const Batch& bt = A.bt;
    ulonglong2* acc = reinterpret_cast<ulonglong2*>(A.acc);
    const long c0 = (long)blockIdx.x * kUcCells;
    const int n = (int)min((long)kUcCells, (long)bt.C - c0);
    const bool first = A.first_frame != 0;
    if (n < kUcCells) {  // the partial last tile: direct reads (the same update)
        for (int i = threadIdx.x; i < n; i += kUcThreads) {
            const int c = (int)(c0 + i);
            const int sc = scene_of(bt.off->cell, bt.S, c);
            const SceneDev& sd = bt.sc[sc];
            const ulonglong2 v = acc[c];
            if (v.x || v.y) acc[c] = make_ulonglong2(0ull, 0ull);
            k3dom_cell_update(sd.p, bt.fp[sc].gamma_dt, c, (double)(long long)v.x * sd.fx_inv,
                              (double)(long long)v.y * sd.fx_inv, A.cs, A.cw, first);
        }
        return;
    }
    float* s_f = reinterpret_cast<float*>(uc_smem);
    float* s_s = s_f + kUcCells;
    float* s_d = s_s + kUcCells;
    int* s_start = reinterpret_cast<int*>(s_d + kUcCells);
    float* s_w = reinterpret_cast<float*>(s_start + kUcCells);
    float* s_vx = s_w + kUcCells;
    float* s_vy = s_vx + kUcCells;
    float* s_vz = s_vy + kUcCells;
    ulonglong2* s_acc = reinterpret_cast<ulonglong2*>(s_vz + kUcCells);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        constexpr uint32_t fb = sizeof(float) * kUcCells;
        constexpr uint32_t total = 8 * fb + sizeof(ulonglong2) * kUcCells;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&bar)), "r"(total)
                     : "memory");
        bulk_load(s_f, A.cs.free_m + c0, fb, &bar);
        bulk_load(s_s, A.cs.static_m + c0, fb, &bar);
        bulk_load(s_d, A.cs.dyn_m + c0, fb, &bar);
        bulk_load(s_start, A.cw.start + c0, fb, &bar);
        bulk_load(s_w, A.cw.sum_w + c0, fb, &bar);
        bulk_load(s_vx, A.cw.sum_wvx + c0, fb, &bar);
        bulk_load(s_vy, A.cw.sum_wvy + c0, fb, &bar);
        bulk_load(s_vz, A.cw.sum_wvz + c0, fb, &bar);
        bulk_load(s_acc, acc + c0, sizeof(ulonglong2) * kUcCells, &bar);
    }
    if (!bar_wait(&bar, kUcMaxPolls)) {
        if (threadIdx.x == 0) atomicOr(&A.status->copy_timeout, 1u);
        bar_wait(&bar, kUcMaxPolls);  // the copies still write this CTA's shared memory
        return;
    }
    for (int i = threadIdx.x; i < kUcCells; i += kUcThreads) {
        const int c = (int)(c0 + i);
        const int sc = scene_of(bt.off->cell, bt.S, c);
        const SceneDev& sd = bt.sc[sc];
        const ulonglong2 v = s_acc[i];
        if (v.x || v.y) acc[c] = make_ulonglong2(0ull, 0ull);
        CellIn in;
        in.m_f = s_f[i];
        in.m_s = s_s[i];
        in.m_d = s_d[i];
        in.start = first ? -1 : s_start[i];
        in.sum_w = s_w[i];
        in.wvx = s_vx[i];
        in.wvy = s_vy[i];
        in.wvz = s_vz[i];
        k3dom_cell_update_in(sd.p, bt.fp[sc].gamma_dt, c, (double)(long long)v.x * sd.fx_inv,
                             (double)(long long)v.y * sd.fx_inv, in, A.cs, A.cw, first);
    }
}

cudaError_t make_kernel_table_texture(RayBuffers& rb, int S) {
    rb.ktex = 0;
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeLinear;
    rd.res.linear.devPtr = rb.ktab;
    rd.res.linear.desc = cudaCreateChannelDesc<float4>();
    rd.res.linear.sizeInBytes = sizeof(float4) * (size_t)kKernelTabEntries * (size_t)S;
    cudaTextureDesc td = {};
    td.readMode = cudaReadModeElementType;  // the stored FP32 values, no filtering
    td.filterMode = cudaFilterModePoint;
    td.addressMode[0] = cudaAddressModeClamp;
    return cudaCreateTextureObject(&rb.ktex, &rd, &td, nullptr);
}

cudaError_t launch_k3dom_update_cells(const Batch& bt, RayBuffers& rb, CellState cs, CellWork cw, DevStatus* status,
                                      cudaStream_t st) {
    const EvArgs A = make_args(bt, rb, cs, cw, false, status);
    ++g_launches;
    const uintptr_t bases = reinterpret_cast<uintptr_t>(cs.free_m) | reinterpret_cast<uintptr_t>(cs.static_m) |
                            reinterpret_cast<uintptr_t>(cs.dyn_m) | reinterpret_cast<uintptr_t>(cw.start) |
                            reinterpret_cast<uintptr_t>(cw.sum_w) | reinterpret_cast<uintptr_t>(cw.sum_wvx) |
                            reinterpret_cast<uintptr_t>(cw.sum_wvy) | reinterpret_cast<uintptr_t>(cw.sum_wvz) |
                            reinterpret_cast<uintptr_t>(rb.acc);
    if ((bases & 15u) == 0) {  // the bulk copies' alignment (cudaMalloc gives 256 bytes)
        k_k3dom_update_cells_bulk<<<div_up(bt.C, kUcCells), kUcThreads, kUcSmem, st>>>(A);
        return cudaGetLastError();
    }
    // one thread per cell: the update is latency bound, so every cell's reads are in flight at once
    k_k3dom_update_cells<<<div_up(bt.C, kBlock), kBlock, 0, st>>>(A);
    return cudaGetLastError();
}

// The DS launches are persistent too: the count pass and the final pass each get one CTA per
// resident slot (the count pass fits 5 CTAs per SM at 47 registers, the final pass 4).
struct DsLaunch {
    int count_blocks, final_blocks;
};

static DsLaunch ds_launch() {
    int dev = 0, sms = 148, per_count = 1, per_final = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_count, k_dsgrid<true>, kEvThreads, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_final, k_dsgrid<false>, kEvThreads, 0);
    return DsLaunch{sms * std::max(1, per_count), sms * std::max(1, per_final)};
}

void k3dom_ds_evidence_blocks(int* count_blocks, int* final_blocks) {
    const DsLaunch L = ds_launch();
    *count_blocks = L.count_blocks;
    *final_blocks = L.final_blocks;
}

cudaError_t launch_ds_evidence(const Batch& bt, RayBuffers& rb, CellState cs, CellWork cw, bool first_frame,
                               DevStatus* status, cudaStream_t st) {
    if (rb.chunk < 32 || rb.chunk > kChunk) return cudaErrorInvalidValue;
    EvArgs A = make_args(bt, rb, cs, cw, first_frame, status);
    const DsLaunch L = ds_launch();
    ++g_launches;
    k_dsgrid<true><<<L.count_blocks, kEvThreads, 0, st>>>(A);
    ++g_launches;
    k_dsgrid<false><<<L.final_blocks, kEvThreads, 0, st>>>(A);
    return cudaGetLastError();
}

long ds_count_bytes(long items) { return items * (long)kMaxTileCells; }

cudaError_t evidence_init() {
    cudaError_t e = cudaFuncSetAttribute(k_bgki<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)bgki_smem_bytes(kChunk));
    if (e != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(k_bgki<8, kSmallWarps * 32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)bgki_smem_bytes(kSmallChunk, kSmallWarps))))
        return e;
    if ((e = cudaFuncSetAttribute(k_bgki<4, kEvThreads, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)bgki_smem_bytes(512, kEvWarps, true))))
        return e;
    if ((e = cudaFuncSetAttribute(k_bgki_sums<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)calib_smem_bytes(kChunk))))
        return e;
    if ((e = cudaFuncSetAttribute(k_bgki_sums<4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)calib_smem_bytes(kCalibChunk, true))))
        return e;
    // 48 KB of copies plus the static barrier: above the default per-CTA limit
    return cudaFuncSetAttribute(k_k3dom_update_cells_bulk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)kUcSmem);
}

}  // namespace k3dom
