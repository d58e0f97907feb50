// internal.h -- launch wrappers shared between the .cu files of the library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace k3dom {

// Kernel launches enqueued by this library (host counter; a frame's count is the difference
// across it). Handles are single-threaded, as the reference's DOM is.
extern long g_launches;

// sort.cu
int scan_u32_tiles(long n);
cudaError_t scan_u32_exclusive(const uint32_t* in, uint32_t* out, long n, uint32_t* tmp,
                               uint32_t* total, cudaStream_t st);
// Same with the element count min(*dn, nmax) read on the device (dn may be nullptr).
cudaError_t scan_u32_exclusive_dn(const uint32_t* in, uint32_t* out, long nmax, const uint32_t* dn,
                                  uint32_t* tmp, uint32_t* total, cudaStream_t st);
int radix_tiles(long n);
long radix_hist_words(long n, int max_bits);
int radix_plan(int key_bits, int* pass_bits);
cudaError_t radix_sort_pairs(const uint32_t* keys, const uint32_t* vals, uint32_t* keys_out,
                             uint32_t* vals_out, uint32_t* alt_k, uint32_t* alt_v, long n,
                             int key_bits, uint32_t* hist, uint32_t* scan_tmp, cudaStream_t st);
cudaError_t radix_sort_pairs_dn(const uint32_t* keys, const uint32_t* vals, uint32_t* keys_out,
                                uint32_t* vals_out, uint32_t* alt_k, uint32_t* alt_v, long nmax,
                                const uint32_t* dn, int key_bits, uint32_t* hist,
                                uint32_t* scan_tmp, cudaStream_t st);
cudaError_t sort_init();

// exactscan.cu: inclusive prefix sums of non-negative floats, exact in 128-bit fixed
// point and rounded once to float.
int exact_scan_tiles(long n);
// Scratch bytes for exact_scan of n elements.
size_t exact_scan_scratch_bytes(long n);
cudaError_t exact_scan_float(const float* in, float* out, long n, void* scratch, cudaStream_t st);
// Same over the concatenation a[0..na) ++ b[0..nb).
cudaError_t exact_scan_float2(const float* a, long na, const float* b, long nb, float* out,
                              void* scratch, cudaStream_t st);

// particles.cu
void launch_predict(const DevParams& p, const FrameParams* fp, Particles a, cudaStream_t st);
void launch_shift_particles(const DevParams& p, Particles a, int mx, int my, int mz,
                            cudaStream_t st);
void launch_gather_segsum(const DevParams& p, Particles a, Particles s,
                          const uint32_t* sorted_keys, const uint32_t* perm, CellWork cw,
                          cudaStream_t st);
void launch_reweight(const DevParams& p, Particles s, const uint32_t* sorted_keys, CellWork cw,
                     cudaStream_t st);
void launch_births(const DevParams& p, const FrameParams* fp, const float* born,
                   const float* born_cum, Particles b, cudaStream_t st);
void launch_init_particles(const DevParams& p, const FrameParams* fp, const float* born_cum,
                           Particles a, cudaStream_t st);
void launch_joint_prepare(const DevParams& p, Particles s, Particles b, float* joint_w,
                          cudaStream_t st);
void launch_draw_keys(const DevParams& p, const FrameParams* fp, uint32_t* keys,
                      cudaStream_t st);
void launch_resample(const DevParams& p, const float* joint_cum, const uint32_t* sorted_draws,
                     Particles s, const uint32_t* sorted_keys, Particles b, Particles out,
                     int* ancestors, float* joint_max_out, cudaStream_t st);
void launch_debug_draws(uint64_t seed, int frame, int stage, long first, long count, float* dst,
                        cudaStream_t st);

// cells.cu
void launch_cells_init(const DevParams& p, CellState cs, CellWork cw, cudaStream_t st);
void launch_map_shift_full(const DevParams& p, CellState src, CellState dst, const int* s_start,
                           const int* s_end, int* d_start, int* d_end, int mx, int my, int mz,
                           cudaStream_t st);
void launch_export_field(const DevParams& p, int field, CellState cs, CellWork cw,
                         const float* born_cum, float* dst, cudaStream_t st);
void launch_export_gridcell(const DevParams& p, CellState cs, CellWork cw, const float* born_cum,
                            void* dst, cudaStream_t st);
void launch_export_mappoints(const DevParams& p, float cx, float cy, float cz, CellState cs,
                             CellWork cw, float* dst, cudaStream_t st);

// evidence.cu
struct RayBuffers {
    float4* ray_a;         // m.x, m.y, m.z, d_m (K3DOM) | |m|^2 (DS)
    float4* ray_b;         // u.x, u.y, u.z, margin (FP32 unit direction)
    double4* ray_c;        // d_m, margin, 1/d_m, 0 in FP64 (K3DOM)
    float4* ktab;          // sparse-kernel table (build_kernel_table)
    uint32_t* counts;      // per ray: number of tiles touched
    uint32_t* offsets;     // exclusive scan of counts
    uint32_t* ekeys;       // entries: tile id
    uint32_t* evals;       // entries: ray id
    uint32_t* ekeys2;      // sorted
    uint32_t* evals2;
    uint32_t* ekeys_alt;
    uint32_t* evals_alt;
    uint32_t* tile_start;  // T+1
    uint32_t* tile_items;  // T: work items per tile
    uint32_t* item_off;    // T+1 work-item offsets per tile
    uint32_t* tile_done;   // T
    unsigned long long* acc;  // 2*C fixed-point accumulators (K3DOM) / DS partials
    uint8_t* ds_counts;    // DS: per (item, cell) hit counts of pass 1
    uint32_t* ds_quota_base;  // DS: item index of a tile's first item
    uint32_t* hist;
    uint32_t* scan_tmp;
    uint32_t* total;       // [0] = entries, [2] = entries kept (0 on overflow)
    long capacity;         // entries
    long ds_count_capacity;
    int max_points;
    int tiles, tx, ty, tz, ntx, nty, ntz;
};
struct EvidenceConfig {
    int tile_x, tile_y, tile_z;  // cells per tile (multiples of 4, 4, 2)
    int chunk;                   // rays per work item
};
long ray_entries_bound(const DevParams& p, const EvidenceConfig& ec, int max_points);
cudaError_t build_ray_lists(const DevParams& p, const FrameParams* fp, const float* xs,
                            const float* ys, const float* zs, RayBuffers& rb, bool ds,
                            DevStatus* status, cudaStream_t st);
cudaError_t launch_k3dom_evidence(const DevParams& p, const FrameParams* fp, RayBuffers& rb,
                                  CellState cs, CellWork cw, bool first_frame,
                                  DevStatus* status, int num_sms, cudaStream_t st);
cudaError_t launch_ds_evidence(const DevParams& p, const FrameParams* fp, RayBuffers& rb,
                               CellState cs, CellWork cw, bool first_frame, DevStatus* status,
                               int num_sms, cudaStream_t st);
cudaError_t evidence_init();
// Host: the sparse-kernel table (512 float4) for sigma, uploaded once per handle.
void build_kernel_table(float sigma, float4* out);
constexpr int kKernelTableSize = 512;

}  // namespace k3dom
