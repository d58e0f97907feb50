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
//  * The scratch (16,384 tile sums of 16 bytes = 256 KiB per device) is shared by every call.
//    Each call overwrites every tile sum it reads, so nothing needs clearing between calls;
//    calls that overlap on the GPU (different streams, no ordering) race on it.
//  * The first call on a device looks up the array's device address (cudaGetSymbolAddress,
//    with that device current) and caches it; make that first call before any stream capture.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/k3dom_b200.h"
#include "common.cuh"
#include "internal.h"
#include "scan.cuh"

namespace k3dom {

constexpr int kNoAllocMaxTiles = 16384;
constexpr long kNoAllocTile = 2048;  // elements per tile of the exact scan (exactscan.cu)
constexpr long kNoAllocMaxElements = (long)kNoAllocMaxTiles * kNoAllocTile;
constexpr int kNoAllocMaxDevices = 64;

// One 128-bit tile sum per tile plus the carry slot exactscan.cu reserves.
static __device__ __align__(256) unsigned char g_noalloc_scratch[(kNoAllocMaxTiles + 1) * sizeof(u128)];

static std::mutex g_noalloc_mu;
static void* g_noalloc_ptr[kNoAllocMaxDevices] = {};

}  // namespace k3dom

using namespace k3dom;

extern "C" k3dom_status k3dom_exact_prefix_sum_noalloc(const float* in, float* out, int64_t n, void* stream) {
    if (n < 0 || (n > 0 && (!in || !out))) return K3DOM_ERR_INVALID_ARGUMENT;
    if (n > kNoAllocMaxElements) return K3DOM_ERR_CAPACITY;
    if (exact_scan_tiles(kNoAllocMaxElements) > kNoAllocMaxTiles || exact_scan_tiles(n) > kNoAllocMaxTiles)
        return K3DOM_ERR_CAPACITY;
    if (n == 0) return K3DOM_OK;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) return K3DOM_ERR_CUDA;
    void* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_ptr[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return K3DOM_ERR_CUDA;
            g_noalloc_ptr[dev] = p;
        }
        scratch = g_noalloc_ptr[dev];
    }
    cudaError_t e = exact_scan_float(in, out, (long)n, scratch, (cudaStream_t)stream);
    return e == cudaSuccess ? K3DOM_OK : K3DOM_ERR_CUDA;
}
