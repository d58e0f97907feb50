// internal.h -- launch wrappers shared between the .cu files of the library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

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
// hist_words / scan_words are the capacities of hist and scan_tmp (radix_hist_words(n, 11) and
// scan_u32_tiles of it suffice for any key width); too small a buffer is refused.
cudaError_t radix_sort_pairs(const uint32_t* keys, const uint32_t* vals, uint32_t* keys_out,
                             uint32_t* vals_out, uint32_t* alt_k, uint32_t* alt_v, long n,
                             int key_bits, uint32_t* hist, long hist_words, uint32_t* scan_tmp,
                             long scan_words, cudaStream_t st);
cudaError_t radix_sort_pairs_dn(const uint32_t* keys, const uint32_t* vals, uint32_t* keys_out,
                                uint32_t* vals_out, uint32_t* alt_k, uint32_t* alt_v, long nmax,
                                const uint32_t* dn, int key_bits, uint32_t* hist, long hist_words,
                                uint32_t* scan_tmp, long scan_words, cudaStream_t st);
cudaError_t sort_init();

// onesweep.cu: the particle sort (one histogram read, then one read and write per 7-bit digit
// with decoupled look-back). A look-back poll loop gives up after max_polls polls and sets
// DevStatus::sort_timeout; skip_tile >= 0 keeps that tile of the first pass from publishing its
// counts (a test hook: every later tile's wait then runs out).
struct SortWait {
    uint32_t max_polls = 1u << 20;
    int skip_tile = -1;
};
int onesweep_plan(int key_bits, int* pass_bits);
long onesweep_scratch_words(long n, int key_bits);
cudaError_t onesweep_init();
cudaError_t onesweep_sort_pairs(const uint32_t* keys, const uint32_t* vals, uint32_t* keys_out, uint32_t* vals_out,
                                uint32_t* alt_k, uint32_t* alt_v, long n, int key_bits, uint32_t* scratch,
                                long scratch_words, DevStatus* ds, const SortWait& wait, cudaStream_t st);
// The same with the element count min(*dn, nmax) read on the device (dn may be nullptr).
cudaError_t onesweep_sort_pairs_dn(const uint32_t* keys, const uint32_t* vals, uint32_t* keys_out, uint32_t* vals_out,
                                   uint32_t* alt_k, uint32_t* alt_v, long nmax, const uint32_t* dn, int key_bits,
                                   uint32_t* scratch, long scratch_words, DevStatus* ds, const SortWait& wait,
                                   cudaStream_t st);

// exactscan.cu: inclusive prefix sums of non-negative floats, exact in 128-bit fixed
// point and rounded once to float.
int exact_scan_tiles(long n);
// Scratch bytes for exact_scan of n elements.
size_t exact_scan_scratch_bytes(long n);
cudaError_t exact_scan_float(const float* in, float* out, long n, void* scratch, cudaStream_t st);
// Same over the concatenation a[0..na) ++ b[0..nb).
cudaError_t exact_scan_float2(const float* a, long na, const float* b, long nb, float* out,
                              void* scratch, cudaStream_t st);

// Segmented exact scan driven by a plan of tiles (each <= 2048 elements, one contiguous input
// and output range, and the index of its segment's first tile).
struct ExactTile {
    float* in;  // writable: a scan may clear its sign-bit inputs in place
    float* out;
    int n;
    int seg_first;
};
// Appends one segment made of `pieces` input ranges, written contiguously from `out`.
void exact_plan_add(std::vector<ExactTile>& plan, float* const* in, const long* n, int pieces, float* out);
size_t exact_plan_scratch_bytes(int ntiles);
// clear_signed: every input with its sign bit set (counted as 0 by the scan) is also set to +0 in
// place, the penalty step of resampling.cu:13-36 folded into the joint weights' scan.
cudaError_t exact_scan_plan(const ExactTile* tiles, int nt, void* scratch, cudaStream_t st, bool clear_signed = false);

// particles.cu
// Prediction reads the structure-of-arrays set a and writes each particle as a 32-byte record
// (x[2i] = px py pz vx, x[2i+1] = vy vz w assoc) plus its cell index a.cell.
void launch_predict(const Batch& bt, Particles a, float4* x, cudaStream_t st);
void launch_pack_records(int n, Particles a, float4* x, cudaStream_t st);
void launch_unpack_records(int n, const float4* x, Particles a, cudaStream_t st);
void launch_shift_particles(int n, Particles a, int mx, int my, int mz, cudaStream_t st);
// Piece sums of one 128-slot range of the sorted particles (gather + segmented sums): the
// range's first piece when its cell began in an earlier range, and its last piece when its cell
// continues into the next range.
struct SegRec {
    double lead[4];   // sum w, w vx, w vy, w vz of the first piece
    double trail[4];  // the same of the last piece
    int lead_end;     // position of the first piece's last particle; -1: it reaches the range's end
    int trail_head;   // position of the last piece's cell head; -1: no such piece
};
long seg_rec_count(long P);
void launch_gather_segsum(const Batch& bt, const float4* x, Particles s, const uint32_t* sorted_keys,
                          const uint32_t* perm, CellWork cw, SegRec* rec, cudaStream_t st);
void launch_reweight(const Batch& bt, Particles s, const uint32_t* sorted_keys, CellWork cw, cudaStream_t st);
void launch_births(const Batch& bt, const float* born, const float* born_cum, Particles b, cudaStream_t st);
void launch_init_particles(const Batch& bt, const float* born_cum, Particles a, cudaStream_t st);
int draw_key_bits(int S);
void launch_draw_keys(const Batch& bt, uint32_t* keys, cudaStream_t st);
long res_bracket_count(long P);
void launch_resample(const Batch& bt, const float* joint_cum, const uint32_t* sorted_draws, Particles s,
                     Particles b, Particles out, int* ancestors, float* joint_max_out, int2* brackets,
                     cudaStream_t st);
void launch_debug_draws(uint64_t seed, int frame, int stage, long first, long count, float* dst,
                        cudaStream_t st);

// cells.cu
void launch_cells_init(const Batch& bt, CellState cs, CellWork cw, cudaStream_t st);
void launch_map_shift_full(const DevParams& p, CellState src, CellState dst, const int* s_start,
                           const int* s_end, int* d_start, int* d_end, int mx, int my, int mz,
                           cudaStream_t st);
// Exports take the scene's own ranges (pointers offset by its cell range); range_base is the
// scene's first sorted particle.
void launch_export_field(const DevParams& p, int field, CellState cs, CellWork cw,
                         const float* born_cum, int range_base, float* dst, cudaStream_t st);
void launch_export_gridcell(const DevParams& p, CellState cs, CellWork cw, const float* born_cum,
                            int range_base, void* dst, cudaStream_t st);
void launch_export_mappoints(const DevParams& p, float cx, float cy, float cz, CellState cs,
                             CellWork cw, float* dst, cudaStream_t st);

// evidence.cu
struct RayBuffers {
    float4* ray_a;         // m.x, m.y, m.z, d_m (K3DOM) | |m|^2 (DS)
    double4* ray_c;        // d_m, margin, 1/d_m, 0 in FP64 (K3DOM)
    float4* ktab;          // per scene: sparse-kernel table with the fixed-point scale folded in
    cudaTextureObject_t ktex;  // ktab read through the texture path (k_bgki), 0 when not made
    uint32_t* counts;      // [kRayThreads * N] tiles touched per point slot (DS) or per thread of a slot
    uint32_t* offsets;     // exclusive scan of counts (DS)
    uint32_t* ekeys;       // entries: global tile id (DS)
    uint32_t* evals;       // entries: point slot (DS)
    uint32_t* ekeys2;      // sorted (DS)
    uint32_t* evals2;      // the lists: point slots grouped by tile (K3DOM: placed, DS: sorted)
    uint32_t* tile_tally;  // T: rays per tile (K3DOM), zero between frames
    uint32_t* block_base;  // [bin_blocks(kRayThreads N)][T]: each binning block's first slot in each tile's range,
                           // relative to the range's start (K3DOM)
    uint32_t* ekeys_alt;
    uint32_t* evals_alt;
    uint32_t* tile_start;  // T+1
    uint32_t* tile_items;  // T: work items per tile
    uint32_t* item_off;    // T+1 work-item offsets per tile
    uint32_t* tile_done;   // T
    unsigned long long* acc;  // 2*C fixed-point accumulators (K3DOM) / DS partials
    uint8_t* ds_counts;    // DS: per (item, cell) neighbour counts of pass 1
    uint32_t* scan_tmp;
    long scan_words;
    uint32_t* os_scratch;  // onesweep sort of the entries by tile
    long os_words;
    uint32_t* total;       // [0] = entries, [2] = entries kept (0 on overflow)
    long capacity;         // entries
    long ds_count_capacity;
    int chunk;             // rays per work item
};
long ray_entries_bound(const DevParams& p, const TileShape& ts, int max_points, float bin_R);
// K3DOM ray lists are placed per tile through block histograms of all T tiles in shared memory
// (48 KB at most); DS lists, and batches with more tiles, are sorted by tile.
constexpr int kPlacedMaxTiles = 12288;
inline bool placed_lists(bool ds, int T) { return !ds && T <= kPlacedMaxTiles; }
constexpr int kBinBlocksMax = 1024;
int bin_blocks(long n);  // blocks of the placed-list passes over n threads
constexpr int kRayThreads = 2;  // threads per ray in the placed-list passes
// Texture object over the S kernel tables (point sampling, FP32 as stored), for k_bgki.
cudaError_t make_kernel_table_texture(RayBuffers& rb, int S);
// Per-scene evidence constants (binning radius, cull radius, fixed-point scale); writes the
// scene's kernel table when ktab is not null.
void fill_scene_evidence(SceneDev& sd, bool ds, float4* ktab);
cudaError_t build_ray_lists(const Batch& bt, const float* xs, const float* ys, const float* zs, RayBuffers& rb,
                            bool ds, DevStatus* status, const SortWait& wait, cudaStream_t st);
cudaError_t launch_k3dom_evidence(const Batch& bt, RayBuffers& rb, CellState cs, CellWork cw, bool first_frame,
                                  DevStatus* status, cudaStream_t st, bool fuse_update = true);
// The cell update of a K3DOM frame whose evidence ran with fuse_update = false.
cudaError_t launch_k3dom_update_cells(const Batch& bt, RayBuffers& rb, CellState cs, CellWork cw, DevStatus* status,
                                      cudaStream_t st);
cudaError_t launch_ds_evidence(const Batch& bt, RayBuffers& rb, CellState cs, CellWork cw, bool first_frame,
                               DevStatus* status, cudaStream_t st);
// CTAs of the K3DOM evidence launch for a chunk size (persistent grid).
int k3dom_evidence_blocks(int chunk);
// CTAs of the DS count pass and final pass (persistent: one per resident slot of each build).
void k3dom_ds_evidence_blocks(int* count_blocks, int* final_blocks);
long ds_count_bytes(long items);
cudaError_t evidence_init();
// Host: the sparse-kernel table for sigma, every value multiplied by scale: 512 intervals and a
// zero entry at u = 1 (513 float4), so an index taken at the support's edge needs no clamp.
void build_kernel_table(float sigma, double scale, float4* out);
constexpr int kKernelTableSize = 513;
// Rays per calibration work item: the largest chunk whose evidence-sums build keeps 4 CTAs per
// SM with its per-region ray lists in shared memory.
constexpr int kCalibChunk = 448;
// Calibration: unit-amplitude kernel and -x f'(x) tables scaled to units of 2^-kCalibShift.
constexpr int kCalibShift = 40;
void build_calib_tables(float4* f_tab, float4* dls_tab);
cudaError_t launch_bgki_sums(const Batch& bt, RayBuffers& rb, const float4* f_tab, const float4* dls_tab,
                             unsigned long long* acc4, DevStatus* status, int num_sms, cudaStream_t st);

}  // namespace k3dom
