// noalloc.cu -- an entry point that allocates nothing: the exact prefix sum of non-negative
// floats (the scan that decides birth slots and resampling ancestors) with its scratch in a
// fixed file-scope device array instead of memory allocated by the handle.
//
// Who needs it: code that may not allocate device memory once it runs -- a real-time
// callback whose memory budget is fixed at start-up, work recorded into a CUDA graph by a
// host framework, or a plugin whose device memory belongs to another allocator. It passes its
// own input and output buffers; the only other memory used is the array below, which every
// GPU that loads this library holds until the process exits.
//
// Limits and rules
//  * n <= kNoAllocMaxElements (33,554,432); larger n returns K3DOM_ERR_CAPACITY, no work.
//  * Exact domain: finite values in [0, 2^23) (-0 counts as 0). There the total stays below
//    2^48, inside the 128-bit fixed point, and every prefix is the correctly rounded exact sum
//    (values below 2^-56 enter truncated to a multiple of 2^-80). An element outside it
//    (negative, NaN, infinite, >= 2^23) is refused on the device: out[i] is NaN for every i
//    from the first refused element on. The call does not synchronise, so it cannot return
//    that refusal as a status.
//  * The scratch (16,384 tile sums of 16 bytes = 256 KiB per device, plus the first-refused
//    index) is shared by every call. Each call resets the index and overwrites every tile sum
//    it reads, so nothing carries over between calls; calls that overlap on the GPU
//    (different streams, no ordering) race on it.
//  * The array's device address is looked up with cudaGetSymbolAddress, with the device
//    current, on the first call in each CUDA context (a device reset or another context on the
//    same device gets a fresh lookup); make that first call before any stream capture.
//  * Its launches are not counted in the handles' per-frame launch counts, and each launch's
//    own error is returned; an earlier, unrelated error left pending by the caller is not
//    consumed.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/k3dom_b200.h"
#include "common.cuh"
#include "fixed128.cuh"
#include "scan.cuh"

namespace k3dom {

constexpr int kNaThreads = 256;
constexpr int kNaItems = 8;
constexpr long kNoAllocTile = kNaThreads * kNaItems;  // elements per tile
constexpr int kNoAllocMaxTiles = 16384;
constexpr long kNoAllocMaxElements = (long)kNoAllocMaxTiles * kNoAllocTile;
constexpr int kNoAllocMaxDevices = 64;
constexpr uint32_t kNoAllocLimitBits = 0x4B000000u;  // 2^23 as float bits

// kNoAllocMaxTiles 128-bit tile sums, then one 16-byte slot holding the index of the first
// refused element (unsigned 64-bit).
static __device__ __align__(256) unsigned char g_noalloc_scratch[(kNoAllocMaxTiles + 1) * sizeof(u128)];

__device__ __forceinline__ bool na_valid(float f) {
    const uint32_t b = __float_as_uint(f);
    const uint32_t mag = b & 0x7FFFFFFFu;
    return mag < kNoAllocLimitBits && (b == mag || mag == 0u);
}

__global__ void na_tile_sums(const float* __restrict__ in, long n, u128* __restrict__ tsum,
                             unsigned long long* __restrict__ first_bad) {
    __shared__ u128 sm[kNaThreads / 32 + 1];
    const long base = (long)blockIdx.x * kNoAllocTile;
    u128 s = 0;
#pragma unroll
    for (int j = 0; j < kNaItems; ++j) {
        const long i = base + (long)j * kNaThreads + threadIdx.x;
        if (i < n) {
            const float f = in[i];
            if (na_valid(f))
                s += to_fixed(f);
            else
                atomicMin(first_bad, (unsigned long long)i);
        }
    }
    u128 tot;
    block_exclusive_scan<u128, kNaThreads>(s, sm, &tot);
    if (threadIdx.x == 0) tsum[blockIdx.x] = tot;
}

__global__ void na_tile_offsets(u128* __restrict__ tsum, int ntiles) {
    __shared__ u128 sm[kNaThreads / 32 + 1];
    u128 carry = 0;
    for (int b = 0; b < ntiles; b += kNaThreads) {
        const int i = b + threadIdx.x;
        const u128 v = (i < ntiles) ? tsum[i] : (u128)0;
        u128 tot;
        const u128 ex = block_exclusive_scan<u128, kNaThreads>(v, sm, &tot);
        if (i < ntiles) tsum[i] = carry + ex;
        carry += tot;
    }
}

__global__ void na_apply(const float* __restrict__ in, long n, const u128* __restrict__ toff,
                         const unsigned long long* __restrict__ first_bad, float* __restrict__ out) {
    __shared__ u128 sm[kNaThreads / 32 + 1];
    const long base = (long)blockIdx.x * kNoAllocTile + (long)threadIdx.x * kNaItems;
    const unsigned long long fb = *first_bad;
    u128 v[kNaItems];
    u128 s = 0;
#pragma unroll
    for (int j = 0; j < kNaItems; ++j) {
        const long i = base + j;
        float f = 0.0f;
        if (i < n) f = in[i];
        v[j] = (i < n && na_valid(f)) ? to_fixed(f) : (u128)0;
        s += v[j];
    }
    u128 tot;
    u128 run = toff[blockIdx.x] + block_exclusive_scan<u128, kNaThreads>(s, sm, &tot);
#pragma unroll
    for (int j = 0; j < kNaItems; ++j) {
        const long i = base + j;
        run += v[j];
        if (i < n) out[i] = (unsigned long long)i >= fb ? __int_as_float(0x7FC00000) : from_fixed(run);
    }
}

// The current CUDA context's unique id, through the driver entry points the runtime exposes
// (no link against the driver library). False when they are unavailable.
typedef CUresult (*PFN_ctx_current)(CUcontext*);
typedef CUresult (*PFN_ctx_id)(CUcontext, unsigned long long*);

static bool current_context_id(unsigned long long* id) {
    static PFN_ctx_current get_cur = nullptr;
    static PFN_ctx_id get_id = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* a = nullptr;
        void* b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) == cudaSuccess &&
            qa == cudaDriverEntryPointSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) == cudaSuccess &&
            qb == cudaDriverEntryPointSuccess) {
            get_cur = reinterpret_cast<PFN_ctx_current>(a);
            get_id = reinterpret_cast<PFN_ctx_id>(b);
        }
    }
    if (!get_cur || !get_id) return false;
    CUcontext ctx = nullptr;
    if (get_cur(&ctx) != CUDA_SUCCESS || !ctx) return false;
    return get_id(ctx, id) == CUDA_SUCCESS;
}

struct NoAllocSlot {
    void* ptr = nullptr;
    unsigned long long ctx = 0;
};

static std::mutex g_noalloc_mu;
static NoAllocSlot g_noalloc_slot[kNoAllocMaxDevices];

// The scratch array's device address in the current context (looked up once per context).
static cudaError_t noalloc_scratch(int dev, void** out) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoAllocSlot& s = g_noalloc_slot[dev];
    unsigned long long id = 0;
    bool have = current_context_id(&id);
    if (have && s.ptr && s.ctx == id) {
        *out = s.ptr;
        return cudaSuccess;
    }
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    if (!p) return cudaErrorInvalidSymbol;
    if (!have) have = current_context_id(&id);  // the lookup may have created the context
    s.ptr = have ? p : nullptr;                  // without a context id nothing is cached
    s.ctx = id;
    *out = p;
    return cudaSuccess;
}

}  // namespace k3dom

using namespace k3dom;

extern "C" k3dom_status k3dom_exact_prefix_sum_noalloc(const float* in, float* out, int64_t n, void* stream) {
    if (n < 0 || (n > 0 && (!in || !out))) return K3DOM_ERR_INVALID_ARGUMENT;
    if (n > kNoAllocMaxElements) return K3DOM_ERR_CAPACITY;
    if (n == 0) return K3DOM_OK;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) return K3DOM_ERR_CUDA;
    void* scratch = nullptr;
    if (noalloc_scratch(dev, &scratch) != cudaSuccess) return K3DOM_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    u128* tsum = reinterpret_cast<u128*>(scratch);
    unsigned long long* first_bad = reinterpret_cast<unsigned long long*>(tsum + kNoAllocMaxTiles);
    const int nt = (int)div_up((long)n, kNoAllocTile);
    long nl = (long)n;
    // every byte 0x7F: an index above any n, i.e. nothing refused yet
    if (cudaMemsetAsync(first_bad, 0x7F, sizeof(unsigned long long), st) != cudaSuccess) return K3DOM_ERR_CUDA;
    void* a1[] = {(void*)&in, (void*)&nl, (void*)&tsum, (void*)&first_bad};
    if (cudaLaunchKernel((const void*)na_tile_sums, dim3(nt), dim3(kNaThreads), a1, 0, st) != cudaSuccess)
        return K3DOM_ERR_CUDA;
    int ntl = nt;
    void* a2[] = {(void*)&tsum, (void*)&ntl};
    if (cudaLaunchKernel((const void*)na_tile_offsets, dim3(1), dim3(kNaThreads), a2, 0, st) != cudaSuccess)
        return K3DOM_ERR_CUDA;
    void* a3[] = {(void*)&in, (void*)&nl, (void*)&tsum, (void*)&first_bad, (void*)&out};
    if (cudaLaunchKernel((const void*)na_apply, dim3(nt), dim3(kNaThreads), a3, 0, st) != cudaSuccess)
        return K3DOM_ERR_CUDA;
    return K3DOM_OK;
}
