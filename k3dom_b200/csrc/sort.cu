// sort.cu -- stable LSD radix sort of (uint32 key, uint32 value) pairs and a u32 scan.
//
// Replaces thrust::sort_by_key on the int cell keys (src/common/dom.cu:175-183), which is
// CUB's stable radix sort; stability is what makes the permutation reproducible (equal
// keys keep their pre-sort order). Each pass is reduce-then-scan: an upsweep histogram per
// 4096-key tile, an exclusive scan of the digit-major histogram matrix, and a downsweep
// that ranks the tile in shared memory (warp match-any) and writes each digit run out
// contiguously. No block waits on another, so nothing spins.
//
// Element counts may live in device memory (`dn`), so a captured graph can sort lists whose
// length is only known on the GPU; kernels are grid-stride over tiles and exit early.
#include <cuda_runtime.h>

#include "common.cuh"
#include "internal.h"
#include "scan.cuh"

namespace k3dom {

long g_launches = 0;

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;  // 2048
constexpr int kGridCap = 148 * 8;

__device__ __forceinline__ long dev_n(long nmax, const uint32_t* dn) {
    return dn ? min((long)*dn, nmax) : nmax;
}

// ---------------------------------------------------------------- u32 exclusive scan
__global__ void scan_u32_tile_sums(const uint32_t* __restrict__ in, long nmax, const uint32_t* dn,
                                   uint32_t* __restrict__ tile_sums) {
    __shared__ uint32_t sm[kScanThreads / 32 + 1];
    const long n = dev_n(nmax, dn);
    const long nt = (n + kScanTile - 1) / kScanTile;
    for (long tile = blockIdx.x; tile < nt; tile += gridDim.x) {
        const long base = tile * kScanTile;
        uint32_t s = 0;
#pragma unroll
        for (int j = 0; j < kScanItems; ++j) {
            long i = base + (long)j * kScanThreads + threadIdx.x;
            if (i < n) s += in[i];
        }
        uint32_t tot;
        block_exclusive_scan<uint32_t, kScanThreads>(s, sm, &tot);
        if (threadIdx.x == 0) tile_sums[tile] = tot;
    }
}

// One block scans the tile sums in place (exclusive) and writes the grand total.
__global__ void scan_u32_tile_offsets(uint32_t* __restrict__ tile_sums, long nmax, const uint32_t* dn,
                                      uint32_t* __restrict__ total) {
    __shared__ uint32_t sm[kScanThreads / 32 + 1];
    const long n = dev_n(nmax, dn);
    const long nt = (n + kScanTile - 1) / kScanTile;
    uint32_t carry = 0;
    for (long b = 0; b < nt; b += kScanThreads) {
        long i = b + threadIdx.x;
        uint32_t v = (i < nt) ? tile_sums[i] : 0u;
        uint32_t tot;
        uint32_t ex = block_exclusive_scan<uint32_t, kScanThreads>(v, sm, &tot);
        if (i < nt) tile_sums[i] = carry + ex;
        carry += tot;
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void scan_u32_apply(const uint32_t* __restrict__ in, long nmax, const uint32_t* dn,
                               const uint32_t* __restrict__ tile_offsets, uint32_t* __restrict__ out) {
    __shared__ uint32_t sm[kScanThreads / 32 + 1];
    const long n = dev_n(nmax, dn);
    const long nt = (n + kScanTile - 1) / kScanTile;
    for (long tile = blockIdx.x; tile < nt; tile += gridDim.x) {
        const long base = tile * kScanTile + (long)threadIdx.x * kScanItems;
        uint32_t v[kScanItems];
        uint32_t s = 0;
#pragma unroll
        for (int j = 0; j < kScanItems; ++j) {
            long i = base + j;
            v[j] = (i < n) ? in[i] : 0u;
            s += v[j];
        }
        uint32_t tot;
        uint32_t ex = block_exclusive_scan<uint32_t, kScanThreads>(s, sm, &tot);
        uint32_t run = tile_offsets[tile] + ex;
#pragma unroll
        for (int j = 0; j < kScanItems; ++j) {
            long i = base + j;
            if (i < n) out[i] = run;
            run += v[j];
        }
    }
}

int scan_u32_tiles(long n) { return div_up(n, kScanTile); }

static int tile_grid(long tiles) { return (int)std::max(1L, std::min(tiles, (long)kGridCap)); }

// Exclusive scan of n u32 values (in may alias out); n = min(*dn, nmax) when dn is given.
// tmp needs scan_u32_tiles(nmax) words. total (optional, device) receives the sum.
cudaError_t scan_u32_exclusive_dn(const uint32_t* in, uint32_t* out, long nmax, const uint32_t* dn,
                                  uint32_t* tmp, uint32_t* total, cudaStream_t st) {
    if (nmax <= 0) return cudaSuccess;
    int nt = scan_u32_tiles(nmax);
    ++g_launches;
    scan_u32_tile_sums<<<tile_grid(nt), kScanThreads, 0, st>>>(in, nmax, dn, tmp);
    ++g_launches;
    scan_u32_tile_offsets<<<1, kScanThreads, 0, st>>>(tmp, nmax, dn, total);
    ++g_launches;
    scan_u32_apply<<<tile_grid(nt), kScanThreads, 0, st>>>(in, nmax, dn, tmp, out);
    return cudaGetLastError();
}

cudaError_t scan_u32_exclusive(const uint32_t* in, uint32_t* out, long n, uint32_t* tmp, uint32_t* total,
                               cudaStream_t st) {
    return scan_u32_exclusive_dn(in, out, n, nullptr, tmp, total, st);
}

// ---------------------------------------------------------------- radix sort
template <int BITS>
__global__ void __launch_bounds__(kSortThreads)
radix_upsweep(const uint32_t* __restrict__ keys, long nmax, const uint32_t* dn, int shift,
              uint32_t* __restrict__ hist, uint32_t* __restrict__ hist_len) {
    constexpr int NB = 1 << BITS;
    __shared__ uint32_t h[NB];
    const long n = dev_n(nmax, dn);
    const long nt = (n + kSortTile - 1) / kSortTile;
    if (blockIdx.x == 0 && threadIdx.x == 0 && hist_len) *hist_len = (uint32_t)(nt << BITS);
    for (long tile = blockIdx.x; tile < nt; tile += gridDim.x) {
        for (int d = threadIdx.x; d < NB; d += kSortThreads) h[d] = 0;
        __syncthreads();
        const long base = tile * kSortTile;
#pragma unroll 4
        for (int j = 0; j < kSortItems; ++j) {
            long i = base + (long)j * kSortThreads + threadIdx.x;
            if (i < n) atomicAdd(&h[(keys[i] >> shift) & (NB - 1)], 1u);
        }
        __syncthreads();
        for (int d = threadIdx.x; d < NB; d += kSortThreads) hist[(long)d * nt + tile] = h[d];
        __syncthreads();
    }
}

template <int BITS>
struct RadixSmem {
    static constexpr int NB = 1 << BITS;
    static constexpr int NW = kSortThreads / 32;
    uint16_t cnt[NW][NB];
    uint32_t digit_start[NB];
    uint32_t global_base[NB];
    uint32_t keys[kSortTile];
    uint32_t vals[kSortTile];
    uint32_t scan_tmp[NW + 1];
};

// vals_in == nullptr: the value is the input position (first pass of an argsort).
// vals_out == nullptr: values are not written (key-only sort).
// CTAs per SM that the shared memory of a BITS-wide pass allows (RadixSmem: 38, 56, 80 KB)
template <int BITS>
struct DownsweepMinBlocks {
    static constexpr int value = BITS <= 8 ? 4 : (BITS <= 10 ? 3 : 2);
};

template <int BITS>
__global__ void __launch_bounds__(kSortThreads, DownsweepMinBlocks<BITS>::value)
radix_downsweep(const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in, long nmax,
                const uint32_t* dn, int shift, const uint32_t* __restrict__ hist_scan,
                uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out) {
    constexpr int NB = 1 << BITS;
    constexpr int NW = kSortThreads / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    RadixSmem<BITS>& S = *reinterpret_cast<RadixSmem<BITS>*>(smem_raw);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const long n = dev_n(nmax, dn);
    const long ntiles = (n + kSortTile - 1) / kSortTile;
    const unsigned lt_mask = (1u << lane) - 1u;

    for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long tbase = tile * kSortTile;
        for (int i = threadIdx.x; i < NW * NB; i += kSortThreads) (&S.cnt[0][0])[i] = 0;
        __syncthreads();

        uint32_t key[kSortItems], val[kSortItems];
        uint16_t rank[kSortItems];
#pragma unroll
        for (int j = 0; j < kSortItems; ++j) {
            long i = tbase + wid * (kSortItems * 32) + j * 32 + lane;
            bool valid = i < n;
            key[j] = valid ? keys_in[i] : 0u;
            val[j] = valid ? (vals_in ? vals_in[i] : (uint32_t)i) : 0u;
            uint32_t d = valid ? ((key[j] >> shift) & (NB - 1)) : 0xFFFFFFFFu;
            unsigned peers = __match_any_sync(0xffffffffu, d);
            int leader = __ffs(peers) - 1;
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
        for (int d = threadIdx.x; d < NB; d += kSortThreads) {
            uint32_t run = 0;
#pragma unroll
            for (int w = 0; w < NW; ++w) {
                uint32_t c = S.cnt[w][d];
                S.cnt[w][d] = (uint16_t)run;
                run += c;
            }
            S.digit_start[d] = run;
        }
        __syncthreads();
        {
            constexpr int PER = (NB + kSortThreads - 1) / kSortThreads;
            uint32_t v[PER];
            uint32_t s = 0;
#pragma unroll
            for (int q = 0; q < PER; ++q) {
                int d = threadIdx.x * PER + q;
                v[q] = (d < NB) ? S.digit_start[d] : 0u;
                s += v[q];
            }
            uint32_t tot;
            uint32_t ex = block_exclusive_scan<uint32_t, kSortThreads>(s, S.scan_tmp, &tot);
#pragma unroll
            for (int q = 0; q < PER; ++q) {
                int d = threadIdx.x * PER + q;
                if (d < NB) {
                    S.digit_start[d] = ex;
                    S.global_base[d] = hist_scan[(long)d * ntiles + tile] - ex;
                }
                ex += v[q];
            }
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kSortItems; ++j) {
            long i = tbase + wid * (kSortItems * 32) + j * 32 + lane;
            if (i < n) {
                uint32_t d = (key[j] >> shift) & (NB - 1);
                uint32_t pos = S.digit_start[d] + S.cnt[wid][d] + rank[j];
                S.keys[pos] = key[j];
                S.vals[pos] = val[j];
            }
        }
        __syncthreads();
        const int valid_n = (int)min((long)kSortTile, n - tbase);
        for (int k = threadIdx.x; k < valid_n; k += kSortThreads) {
            uint32_t kk = S.keys[k];
            uint32_t d = (kk >> shift) & (NB - 1);
            uint32_t dest = S.global_base[d] + k;
            if (keys_out) keys_out[dest] = kk;
            if (vals_out) vals_out[dest] = S.vals[k];
        }
        __syncthreads();
    }
}

int radix_tiles(long n) { return div_up(n, kSortTile); }
long radix_hist_words(long n, int max_bits) { return ((long)radix_tiles(n) << max_bits) + 1; }

template <int BITS>
static cudaError_t radix_pass(const uint32_t* kin, const uint32_t* vin, uint32_t* kout, uint32_t* vout,
                              long nmax, const uint32_t* dn, int shift, uint32_t* hist, uint32_t* scan_tmp,
                              cudaStream_t st) {
    const int nt = radix_tiles(nmax);
    const long hn = (long)nt << BITS;
    // the last word of hist holds the live histogram length (device count case)
    uint32_t* hist_len = hist + hn;
    ++g_launches;
    radix_upsweep<BITS><<<tile_grid(nt), kSortThreads, 0, st>>>(kin, nmax, dn, shift, hist, dn ? hist_len : nullptr);
    cudaError_t e = scan_u32_exclusive_dn(hist, hist, hn, dn ? hist_len : nullptr, scan_tmp, nullptr, st);
    if (e != cudaSuccess) return e;
    ++g_launches;
    radix_downsweep<BITS><<<tile_grid(nt), kSortThreads, sizeof(RadixSmem<BITS>), st>>>(kin, vin, nmax, dn, shift,
                                                                                       hist, kout, vout);
    return cudaGetLastError();
}

cudaError_t sort_init() {
    cudaError_t e;
    e = cudaFuncSetAttribute(radix_downsweep<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(RadixSmem<8>));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(radix_downsweep<10>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(RadixSmem<10>));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(radix_downsweep<11>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)sizeof(RadixSmem<11>));
    return e;
}

static cudaError_t radix_pass_bits(int bits, const uint32_t* kin, const uint32_t* vin, uint32_t* kout,
                                   uint32_t* vout, long nmax, const uint32_t* dn, int shift, uint32_t* hist,
                                   uint32_t* scan_tmp, cudaStream_t st) {
    if (bits <= 8) return radix_pass<8>(kin, vin, kout, vout, nmax, dn, shift, hist, scan_tmp, st);
    if (bits <= 10) return radix_pass<10>(kin, vin, kout, vout, nmax, dn, shift, hist, scan_tmp, st);
    return radix_pass<11>(kin, vin, kout, vout, nmax, dn, shift, hist, scan_tmp, st);
}

// Split key_bits into passes of at most 11 bits, as even as possible.
int radix_plan(int key_bits, int* pass_bits) {
    if (key_bits <= 0) key_bits = 1;
    int np = (key_bits + 10) / 11;
    int base = key_bits / np, extra = key_bits % np;
    for (int p = 0; p < np; ++p) pass_bits[p] = base + (p < extra ? 1 : 0);
    return np;
}

// Stable sort by the low key_bits bits. The result lands in keys_out / vals_out; alt_k /
// alt_v are ping-pong buffers (unused for a single pass). vals == nullptr sorts an
// identity payload (argsort); vals_out == nullptr sorts keys only.
// hist_words / scan_words: capacity of hist and scan_tmp; a call whose passes would need more
// is refused (cudaErrorInvalidValue) before anything is launched.
cudaError_t radix_sort_pairs_dn(const uint32_t* keys, const uint32_t* vals, uint32_t* keys_out,
                                uint32_t* vals_out, uint32_t* alt_k, uint32_t* alt_v, long nmax,
                                const uint32_t* dn, int key_bits, uint32_t* hist, long hist_words,
                                uint32_t* scan_tmp, long scan_words, cudaStream_t st) {
    if (nmax <= 0) return cudaSuccess;
    int pb[4];
    const int np = radix_plan(key_bits, pb);
    for (int p = 0; p < np; ++p) {
        const int tb = pb[p] <= 8 ? 8 : (pb[p] <= 10 ? 10 : 11);  // template width of the pass
        const long hn = (long)radix_tiles(nmax) << tb;
        if (hn + 1 > hist_words || scan_u32_tiles(hn) > scan_words) return cudaErrorInvalidValue;
    }
    const uint32_t* ck = keys;
    const uint32_t* cv = vals;
    int shift = 0;
    for (int p = 0; p < np; ++p) {
        const bool to_out = ((np - 1 - p) % 2) == 0;
        uint32_t* ok = to_out ? keys_out : alt_k;
        uint32_t* ov = vals_out ? (to_out ? vals_out : alt_v) : nullptr;
        cudaError_t e = radix_pass_bits(pb[p], ck, cv, ok, ov, nmax, dn, shift, hist, scan_tmp, st);
        if (e != cudaSuccess) return e;
        ck = ok;
        cv = ov;
        shift += pb[p];
    }
    return cudaSuccess;
}

cudaError_t radix_sort_pairs(const uint32_t* keys, const uint32_t* vals, uint32_t* keys_out, uint32_t* vals_out,
                             uint32_t* alt_k, uint32_t* alt_v, long n, int key_bits, uint32_t* hist,
                             long hist_words, uint32_t* scan_tmp, long scan_words, cudaStream_t st) {
    return radix_sort_pairs_dn(keys, vals, keys_out, vals_out, alt_k, alt_v, n, nullptr, key_bits, hist, hist_words,
                               scan_tmp, scan_words, st);
}

}  // namespace k3dom
