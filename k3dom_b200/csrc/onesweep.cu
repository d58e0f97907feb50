// onesweep.cu -- stable LSD radix sort of (uint32 key, uint32 value) pairs in one pass over the
// data per digit ("onesweep"): the particle assignment's sort by cell.
//
// Replaces thrust::sort_by_key on the int cell keys (src/common/dom.cu:175-183), CUB's stable
// radix sort; stability (equal keys keep their pre-sort order) makes the permutation
// reproducible. The digit histograms of every pass come from one read of the keys; then each
// pass reads every (key, value) once and writes it once:
//  * a CTA takes the next 4096-key tile from a counter (tiles are handed out in launch order,
//    so every earlier tile belongs to a CTA that is already running or done), ranks its keys
//    stably in shared memory (warp match-any, warps in order), publishes its per-digit counts,
//    and finds the number of earlier keys of each digit by decoupled look-back over the
//    earlier tiles' published counts (aggregate or inclusive prefix), then publishes its
//    inclusive prefix and writes each digit run out contiguously;
//  * a look-back that finds an earlier tile's counts not yet published polls again, at most
//    `max_polls` times; past that it records a timeout in the device status and the CTA returns
//    without writing (the host then reports K3DOM_ERR_TIMEOUT). No wait is unbounded. Every
//    position a CTA writes is still correct (an abandoned tile published its counts before its
//    look-back, so later tiles count past it), so the output holds the keys and values of the
//    completed tiles and in-range old contents elsewhere; the later passes then write nothing.
// Digits of up to 8 bits, a key of b bits taking ceil(b / 8) passes of (nearly) equal width:
// the 21-bit cell keys of 2^21 voxels three passes of 7 bits, the 24-bit resampling draws three
// of 8 (four passes of 6 before: the draws' sort runs beside the particle sort and slowed it);
// up to 256 digits per tile keep the runs long enough for coalesced writes. The element count
// may live in device memory (`dn`, capped at nmax): the grid and scratch are sized for nmax,
// CTAs whose tile lies past the live count return, and since tiles are handed out in order no
// CTA waits on one of them. The same
// sort orders the resampling draws (keys only) and the ray lists (tile of each entry, stable so
// each tile keeps its rays in input order).
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "internal.h"
#include "scan.cuh"

namespace k3dom {

constexpr int kOsThreads = 256;
constexpr int kOsItems = 16;
constexpr int kOsTile = kOsThreads * kOsItems;  // 4096 keys
constexpr int kOsMaxBits = 8;
constexpr int kOsDigits = 1 << kOsMaxBits;
constexpr int kOsMaxPasses = 5;                 // up to 35-bit keys (uint32 keys need at most 5)
constexpr uint32_t kOsAgg = 1u << 30;           // published: this tile's count of the digit
constexpr uint32_t kOsInc = 2u << 30;           // published: inclusive prefix through this tile
constexpr uint32_t kOsValue = (1u << 30) - 1u;
constexpr int kOsHistBlocks = 148 * 4;
constexpr int kOsWindow = 16;  // predecessor statuses read per look-back step
constexpr int kOsPassBlocks = 3;  // CTAs per SM of a pass (its registers: tile loads in flight)

// scratch layout (uint32 words): counters [kOsMaxPasses + 1] | histograms [passes][kOsDigits] |
// digit offsets [passes][kOsDigits] | tile status [passes][tiles][kOsDigits]
struct OsScratch {
    uint32_t* counters;  // tile counter of each pass, then the histogram CTAs' done counter
    uint32_t* hist;
    uint32_t* digit_off;
    uint32_t* status;
};

static OsScratch os_layout(uint32_t* base, int passes) {
    OsScratch s;
    s.counters = base;
    s.hist = base + kOsMaxPasses + 1;
    s.digit_off = s.hist + (long)passes * kOsDigits;
    s.status = s.digit_off + (long)passes * kOsDigits;
    return s;
}

int onesweep_plan(int key_bits, int* pass_bits) {
    if (key_bits <= 0) key_bits = 1;
    const int np = (key_bits + kOsMaxBits - 1) / kOsMaxBits;
    const int base = key_bits / np, extra = key_bits % np;
    for (int p = 0; p < np; ++p) pass_bits[p] = base + (p < extra ? 1 : 0);
    return np;
}

long onesweep_scratch_words(long n, int key_bits) {
    int pb[kOsMaxPasses];
    const int np = onesweep_plan(key_bits, pb);
    const long tiles = div_up(std::max(n, 1L), (long)kOsTile);
    return (kOsMaxPasses + 1) + 2L * np * kOsDigits + (long)np * tiles * kOsDigits;
}

// A tile's status word carries its flag and its count together and guards no other data, so
// relaxed (coherent, unordered) accesses at device scope suffice.
__device__ __forceinline__ uint32_t ld_status(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_status(uint32_t* p, uint32_t v) {
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

struct OsPasses {
    int np;
    int shift[kOsMaxPasses];
    int bits[kOsMaxPasses];
};

__device__ __forceinline__ long os_count(long nmax, const uint32_t* dn) {
    return dn ? min((long)*dn, nmax) : nmax;
}

// Digit histograms of every pass in one read of the keys; the last CTA to finish turns them
// into each pass's exclusive digit offsets (no CTA waits on another). Each thread counts a run of
// kOsHistRun consecutive keys and adds each digit's run length with one shared atomic: the
// particles keep their cell order from frame to frame, so their keys arrive nearly sorted and
// one atomic per key would serialise on a few shared counters.
constexpr int kOsHistRun = 8;

__global__ void __launch_bounds__(kOsThreads) os_hist(const uint32_t* __restrict__ keys, long nmax,
                                                      const uint32_t* dn, OsPasses ps, OsScratch sc) {
    __shared__ uint32_t h[kOsMaxPasses][kOsDigits];
    __shared__ bool last;
    const long n = os_count(nmax, dn);
    for (int i = threadIdx.x; i < ps.np * kOsDigits; i += kOsThreads) (&h[0][0])[i] = 0;
    __syncthreads();
    const long stride = (long)gridDim.x * kOsThreads * kOsHistRun;
    const bool vec = (reinterpret_cast<uintptr_t>(keys) & 15u) == 0;
    for (long base = ((long)blockIdx.x * kOsThreads + threadIdx.x) * kOsHistRun; base < n; base += stride) {
        uint32_t k[kOsHistRun];
        if (vec && base + kOsHistRun <= n) {  // 16-byte aligned: base is a multiple of 8 keys
            const uint4 a = __ldg(reinterpret_cast<const uint4*>(keys + base));
            const uint4 b = __ldg(reinterpret_cast<const uint4*>(keys + base) + 1);
            k[0] = a.x; k[1] = a.y; k[2] = a.z; k[3] = a.w;
            k[4] = b.x; k[5] = b.y; k[6] = b.z; k[7] = b.w;
        } else {
#pragma unroll
            for (int i = 0; i < kOsHistRun; ++i) k[i] = base + i < n ? keys[base + i] : 0u;
        }
        const int m = (int)min((long)kOsHistRun, n - base);
#pragma unroll
        for (int p = 0; p < kOsMaxPasses; ++p) {
            if (p >= ps.np) break;
            const uint32_t mask = (1u << ps.bits[p]) - 1u;
            const int sh = ps.shift[p];
            uint32_t cur = (k[0] >> sh) & mask, run = 1;
#pragma unroll
            for (int i = 1; i < kOsHistRun; ++i) {
                if (i >= m) break;
                const uint32_t d = (k[i] >> sh) & mask;
                if (d != cur) {
                    atomicAdd(&h[p][cur], run);
                    cur = d;
                    run = 0;
                }
                ++run;
            }
            atomicAdd(&h[p][cur], run);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < ps.np * kOsDigits; i += kOsThreads) {
        const uint32_t v = (&h[0][0])[i];
        if (v) atomicAdd(&sc.hist[i], v);
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(&sc.counters[kOsMaxPasses], 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    __shared__ uint32_t tmp[kOsThreads / 32 + 1];
    for (int p = 0; p < ps.np; ++p) {  // kOsDigits <= kOsThreads: one digit per thread
        const int d = threadIdx.x;
        const uint32_t v = d < kOsDigits ? __ldcg(&sc.hist[p * kOsDigits + d]) : 0u;
        uint32_t tot;
        const uint32_t ex = block_exclusive_scan<uint32_t, kOsThreads>(v, tmp, &tot);
        if (d < kOsDigits) sc.digit_off[p * kOsDigits + d] = ex;
    }
}

struct OsSmem {
    uint16_t cnt[kOsThreads / 32][kOsDigits];
    uint32_t digit_start[kOsDigits];
    uint32_t global_base[kOsDigits];
    uint32_t keys[kOsTile];
    uint32_t vals[kOsTile];
    uint32_t scan_tmp[kOsThreads / 32 + 1];
    uint32_t tile;
};

// One pass of BITS bits at `shift`. vals_in == nullptr: the value is the input position (the
// first pass of an argsort). vals_out == nullptr: keys only.
template <int BITS>
__global__ void __launch_bounds__(kOsThreads, kOsPassBlocks)
os_pass(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in, long nmax, const uint32_t* dn,
        int shift, int pass, OsScratch sc, uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out,
        DevStatus* ds, uint32_t max_polls, int skip_tile) {
    constexpr int NB = 1 << BITS;
    constexpr int NW = kOsThreads / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    OsSmem& S = *reinterpret_cast<OsSmem*>(smem_raw);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    const long cap_tiles = (nmax + kOsTile - 1) / kOsTile;  // the grid and the status layout
    const long n = os_count(nmax, dn);
    const long ntiles = (n + kOsTile - 1) / kOsTile;        // live tiles
    // after a timeout in an earlier pass this pass's input is incomplete, so its digit counts no
    // longer match the histograms: write nothing (every output slot keeps an in-range value)
    if (pass > 0 && *(volatile unsigned int*)&ds->sort_timeout) return;
    uint32_t* status = sc.status + ((long)pass * cap_tiles) * kOsDigits;
    // persistent CTAs: each takes tiles from the counter until none is left
    for (;;) {
        if (threadIdx.x == 0) S.tile = atomicAdd(&sc.counters[pass], 1u);
        // the counters' rows are kOsDigits wide whatever the pass's width: clear them all
        for (int i = threadIdx.x; i < NW * kOsDigits; i += kOsThreads) (&S.cnt[0][0])[i] = 0;
        __syncthreads();
        const long tile = S.tile;
        if (tile >= ntiles) return;  // no live tile left
        const long tbase = tile * kOsTile;

        // stable rank within the tile: warp w holds keys [w*512, w*512 + 512) in (item, lane) order;
        // every load of the tile is issued before the ranking
        uint32_t key[kOsItems], val[kOsItems];
        uint16_t rank[kOsItems];
    #pragma unroll
        for (int j = 0; j < kOsItems; ++j) {
            const long i = tbase + wid * (kOsItems * 32) + j * 32 + lane;
            const bool valid = i < n;
            key[j] = valid ? keys_in[i] : 0u;
            val[j] = valid ? (vals_in ? vals_in[i] : (uint32_t)i) : 0u;
        }
    #pragma unroll
        for (int j = 0; j < kOsItems; ++j) {
            const long i = tbase + wid * (kOsItems * 32) + j * 32 + lane;
            const bool valid = i < n;
            const uint32_t d = valid ? ((key[j] >> shift) & (NB - 1)) : 0xFFFFFFFFu;
            const unsigned peers = __match_any_sync(0xffffffffu, d);
            const int leader = __ffs(peers) - 1;
            uint32_t base = 0;
            if (valid && lane == leader) {
                base = S.cnt[wid][d];
                S.cnt[wid][d] = (uint16_t)(base + __popc(peers));
            }
            base = __shfl_sync(0xffffffffu, base, leader);
            rank[j] = (uint16_t)(base + __popc(peers & lt_mask));
            __syncwarp();
        }
        __syncthreads();
        // per digit: warp offsets (exclusive over warps) and the tile's count
        uint32_t count = 0;
        if (threadIdx.x < NB) {
            const int d = threadIdx.x;
    #pragma unroll
            for (int w = 0; w < NW; ++w) {
                const uint32_t c = S.cnt[w][d];
                S.cnt[w][d] = (uint16_t)count;
                count += c;
            }
            if (tile != skip_tile) st_status(&status[tile * kOsDigits + d], kOsAgg | count);
        }
        // tile-local digit starts
        {
            uint32_t tot;
            const uint32_t ex = block_exclusive_scan<uint32_t, kOsThreads>(count, S.scan_tmp, &tot);
            if (threadIdx.x < NB) S.digit_start[threadIdx.x] = ex;
        }
        __syncthreads();
        // the tile in digit order in shared memory (positions need no earlier tile), so the keys
        // leave the registers before the look-back
    #pragma unroll
        for (int j = 0; j < kOsItems; ++j) {
            const long i = tbase + wid * (kOsItems * 32) + j * 32 + lane;
            if (i < n) {
                const uint32_t d = (key[j] >> shift) & (NB - 1);
                const uint32_t pos = S.digit_start[d] + S.cnt[wid][d] + rank[j];
                S.keys[pos] = key[j];
                S.vals[pos] = val[j];
            }
        }
        __syncthreads();
        // decoupled look-back: keys of this digit in all earlier tiles. The statuses of kOsWindow
        // predecessors are read at once (independent loads) and summed in order up to the first
        // inclusive prefix; a predecessor not yet published ends the step there and is polled again.
        // Tiles that start together publish only their counts at first, so a walk of one tile per
        // dependent load would grow with the tile's distance from the last inclusive prefix.
        bool timed_out = false;
        if (threadIdx.x < NB) {
            const int d = threadIdx.x;
            uint32_t excl = 0;
            uint32_t polls = 0;
            long j = tile - 1;
            while (j >= 0) {
                uint32_t st_w[kOsWindow];
    #pragma unroll
                for (int w = 0; w < kOsWindow; ++w)
                    st_w[w] = (j - w >= 0) ? ld_status(&status[(j - w) * kOsDigits + d]) : kOsInc;
                int used = 0;
                bool done = false;
    #pragma unroll
                for (int w = 0; w < kOsWindow; ++w) {
                    if (done || used < w) continue;          // stopped at an earlier entry of the window
                    if ((st_w[w] & ~kOsValue) == 0u) continue;  // not yet published: poll it again
                    excl += st_w[w] & kOsValue;               // tiles before 0 read as an empty prefix
                    used = w + 1;
                    if (st_w[w] & kOsInc) done = true;
                }
                if (done) break;
                if (used == 0) {
                    if (polls++ >= max_polls) {
                        timed_out = true;
                        break;
                    }
                    __nanosleep(64);
                }
                j -= used;
            }
            if (!timed_out && tile != skip_tile) st_status(&status[tile * kOsDigits + d], kOsInc | (excl + count));
            S.global_base[d] = sc.digit_off[pass * kOsDigits + d] + excl - S.digit_start[d];
        }
        if (__syncthreads_or(timed_out)) {
            if (threadIdx.x == 0) atomicOr(&ds->sort_timeout, 1u);
            return;
        }
        const int valid_n = (int)min((long)kOsTile, n - tbase);
        for (int k = threadIdx.x; k < valid_n; k += kOsThreads) {
            const uint32_t kk = S.keys[k];
            const uint32_t d = (kk >> shift) & (NB - 1);
            const uint32_t dest = S.global_base[d] + k;
            if (keys_out) keys_out[dest] = kk;
            if (vals_out) vals_out[dest] = S.vals[k];
        }
        __syncthreads();  // the shared tile is reused by the next iteration
    }
}

template <int BITS>
static cudaError_t os_launch(const uint32_t* kin, const uint32_t* vin, long nmax, const uint32_t* dn, int shift,
                             int pass, OsScratch sc, uint32_t* kout, uint32_t* vout, DevStatus* ds,
                             uint32_t max_polls, int skip_tile, cudaStream_t st) {
    // persistent grid: at most one CTA per resident slot (tiles are handed out by the counter, in
    // order, so a CTA only ever waits on tiles that running CTAs hold or have finished)
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, os_pass<BITS>, kOsThreads, sizeof(OsSmem));
    const long grid = std::min((long)div_up(nmax, (long)kOsTile), (long)sms * std::max(per_sm, 1));
    ++g_launches;
    os_pass<BITS><<<(unsigned)grid, kOsThreads, sizeof(OsSmem), st>>>(kin, vin, nmax, dn, shift, pass, sc, kout,
                                                                       vout, ds, max_polls, skip_tile);
    return cudaGetLastError();
}

cudaError_t onesweep_init() {
    cudaError_t e = cudaSuccess;
    for (auto f : {os_pass<1>, os_pass<2>, os_pass<3>, os_pass<4>, os_pass<5>, os_pass<6>, os_pass<7>})
        if ((e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(OsSmem))))
            return e;
    return e;
}

cudaError_t onesweep_sort_pairs_dn(const uint32_t* keys, const uint32_t* vals, uint32_t* keys_out, uint32_t* vals_out,
                                   uint32_t* alt_k, uint32_t* alt_v, long n, const uint32_t* dn, int key_bits,
                                   uint32_t* scratch, long scratch_words, DevStatus* ds, const SortWait& wait,
                                   cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    if (n > (long)kOsValue || !ds) return cudaErrorInvalidValue;
    OsPasses ps;
    ps.np = onesweep_plan(key_bits, ps.bits);
    if (ps.np > kOsMaxPasses) return cudaErrorInvalidValue;
    if (onesweep_scratch_words(n, key_bits) > scratch_words) return cudaErrorInvalidValue;
    int shift = 0;
    for (int p = 0; p < ps.np; ++p) {
        ps.shift[p] = shift;
        shift += ps.bits[p];
    }
    const OsScratch sc = os_layout(scratch, ps.np);
    cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(uint32_t) * (size_t)onesweep_scratch_words(n, key_bits), st);
    if (e != cudaSuccess) return e;
    ++g_launches;
    const long hist_grid = std::min((long)kOsHistBlocks, (long)div_up(n, (long)kOsThreads));
    os_hist<<<(unsigned)hist_grid, kOsThreads, 0, st>>>(keys, n, dn, ps, sc);
    const uint32_t* ck = keys;
    const uint32_t* cv = vals;
    for (int p = 0; p < ps.np; ++p) {
        const bool to_out = ((ps.np - 1 - p) % 2) == 0;
        uint32_t* ok = to_out ? keys_out : alt_k;
        uint32_t* ov = vals_out ? (to_out ? vals_out : alt_v) : nullptr;
        const int skip = p == 0 ? wait.skip_tile : -1;
        switch (ps.bits[p]) {
            case 1: e = os_launch<1>(ck, cv, n, dn, ps.shift[p], p, sc, ok, ov, ds, wait.max_polls, skip, st); break;
            case 2: e = os_launch<2>(ck, cv, n, dn, ps.shift[p], p, sc, ok, ov, ds, wait.max_polls, skip, st); break;
            case 3: e = os_launch<3>(ck, cv, n, dn, ps.shift[p], p, sc, ok, ov, ds, wait.max_polls, skip, st); break;
            case 4: e = os_launch<4>(ck, cv, n, dn, ps.shift[p], p, sc, ok, ov, ds, wait.max_polls, skip, st); break;
            case 5: e = os_launch<5>(ck, cv, n, dn, ps.shift[p], p, sc, ok, ov, ds, wait.max_polls, skip, st); break;
            case 6: e = os_launch<6>(ck, cv, n, dn, ps.shift[p], p, sc, ok, ov, ds, wait.max_polls, skip, st); break;
            case 7: e = os_launch<7>(ck, cv, n, dn, ps.shift[p], p, sc, ok, ov, ds, wait.max_polls, skip, st); break;
            default: e = os_launch<8>(ck, cv, n, dn, ps.shift[p], p, sc, ok, ov, ds, wait.max_polls, skip, st); break;
        }
        if (e != cudaSuccess) return e;
        ck = ok;
        cv = ov;
    }
    return cudaSuccess;
}

cudaError_t onesweep_sort_pairs(const uint32_t* keys, const uint32_t* vals, uint32_t* keys_out, uint32_t* vals_out,
                                uint32_t* alt_k, uint32_t* alt_v, long n, int key_bits, uint32_t* scratch,
                                long scratch_words, DevStatus* ds, const SortWait& wait, cudaStream_t st) {
    return onesweep_sort_pairs_dn(keys, vals, keys_out, vals_out, alt_k, alt_v, n, nullptr, key_bits, scratch,
                                  scratch_words, ds, wait, st);
}

}  // namespace k3dom
