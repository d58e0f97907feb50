// common.cuh -- device-side types shared by the K3DOM B200 kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "draws.cuh"

namespace k3dom {

constexpr int kBlock = 256;

// Constant, per-handle parameters (DOM_c::Params after the node's unit conversions,
// include/common/dom.h:19-52), passed to kernels by value.
struct DevParams {
    int G, Gz, C;        // grid_size, grid_size_z, grid_cell_count (src/common/dom.cu:30-31)
    int P, B;            // particle_count, new_born_particle_count
    float res, size, size_z;
    float mass_scale, p_S, noise_pos, noise_vel, p_B, stddev_vel, init_max_vel, min_vel;
    float prior_free, prior_static, prior_dynamic, prior_occ;
    float sigma, ls, gamma;
    float max_range, meas_occ_stddev, window_radius;
    float p_A, likelihood;  // constant 0 and 1 in both variants (init.cu:32-33)
    uint64_t seed;
    int variant;            // 0 = K3DOM, 1 = DS-PHD/MIB
};

constexpr int kMaxScenes = 64;

// Evidence tiling of one scene: tiles of tx x ty x tz cells (multiples of 4, 4, 2), each cut
// into 4x4x2-cell sub-blocks.
struct TileShape {
    int tx, ty, tz, ntx, nty, ntz, nsbx, nsby;
};

// Per-scene constants in device memory. Every scene of a batch owns contiguous ranges of the
// concatenated cell, particle, birth, joint-weight, point and tile arrays.
struct SceneDev {
    DevParams p;
    TileShape ts;
    int cell_off, part_off, birth_off, joint_off, point_off, tile_off;
    int n_tiles, max_points;
    float bin_R;    // ray-binning support radius [cells]
    float cull_r2;   // DS: squared cull radius around a sub-block centroid [m^2]
    float wr2;       // DS window radius squared [m^2]
    float cull_ls2;  // K3DOM: squared support radius of the sub-block cull, ls plus slack [m^2]
    double fx_inv;   // K3DOM evidence: value = fixed-point integer * fx_inv
};

// Range starts of every scene, entry S = the total (device memory).
struct SceneOffsets {
    int part[kMaxScenes + 1];
    int birth[kMaxScenes + 1];
    int joint[kMaxScenes + 1];
    int cell[kMaxScenes + 1];
    int point[kMaxScenes + 1];
    int tile[kMaxScenes + 1];
};

// Per-frame scalars, resident in device memory so a captured graph can be replayed.
struct FrameParams {
    float dt;
    double gamma_dt;  // gamma^dt of the scene (the prediction's decay), FP64
    float sensor_x, sensor_y, sensor_z;  // sensor position minus map centre [m]
    int n_points;
    uint32_t frame;
    int shift_x, shift_y, shift_z;       // pending particle shift (voxels), applied in predict
    int shift_pending;
    uint64_t seed;
    // optional rigid transform of the scene's points into the map-aligned sensor frame
    // (p' = R p + t), applied where the points are read; has_transform = 0: points as given
    float rot[9];   // row-major
    float trans[3];
    int has_transform;
};

// R p + t in FP32 in the written order, without contraction (a CPU restatement with the same
// operation order reproduces it bit for bit).
__device__ __forceinline__ void apply_transform(const FrameParams& f, float* x, float* y, float* z) {
    const float a = *x, b = *y, c = *z;
    *x = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(f.rot[0], a), __fmul_rn(f.rot[1], b)), __fmul_rn(f.rot[2], c)), f.trans[0]);
    *y = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(f.rot[3], a), __fmul_rn(f.rot[4], b)), __fmul_rn(f.rot[5], c)), f.trans[1]);
    *z = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(f.rot[6], a), __fmul_rn(f.rot[7], b)), __fmul_rn(f.rot[8], c)), f.trans[2]);
}

// The batch as the kernels see it: S scenes, their totals and per-scene tables.
struct Batch {
    int S, variant;
    int P, B, C, N, T;  // total particles, births, cells, point slots, tiles
    const SceneDev* sc;
    const FrameParams* fp;
    const SceneOffsets* off;
};

// Scene owning element i of a concatenated range: the last s with off[s] <= i.
__device__ __forceinline__ int scene_of(const int* off, int S, int i) {
    int lo = 0, hi = S;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (off[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

// Per-handle device status words.
struct DevStatus {
    unsigned long long nonfinite_points;
    unsigned long long ray_entries;
    unsigned long long work_items;
    unsigned int overflow;
    unsigned int work_counter;  // dynamic work queue of the evidence kernels
    unsigned int work_counter2;
    unsigned int nonfinite_frame;  // points skipped as non-finite in the last frame's binning
    unsigned long long kernel_evals;  // in-support sparse-kernel evaluations of the last frame
    unsigned int sort_timeout;        // a bounded look-back wait of the particle sort gave up
    unsigned int copy_timeout;        // a bounded wait for a bulk copy gave up (its cells skipped)
};

// Particle set, SoA (ParticlesSoA, include/common/dom_types.h:76-167; post_weight is
// never stored: likelihood is the constant 1).
struct Particles {
    float *px, *py, *pz, *vx, *vy, *vz, *w;
    int* cell;
    uint8_t* assoc;
};

// Per-cell persistent state that moves with the map (GridCell fields, dom_types.h:12-45).
struct CellState {
    float *free_m, *static_m, *dyn_m, *occ_m, *pers_m, *pred_m, *born_m, *mvx, *mvy, *mvz;
};

// Per-frame per-cell work arrays.
struct CellWork {
    int* start;     // first sorted particle of the cell, -1 when empty
    int* end;       // last sorted particle, -1 when empty
    float* sum_w;   // sum of predicted weights (dom_types.h weight)
    float* sum_wvx; // sum of weight * velocity
    float* sum_wvy;
    float* sum_wvz;
    float* factor;  // per-particle reweight factor p_A mu_A l + (1-p_A) mu_UA
    float* divisor; // DS: in-place normalisation divisor (1 when none)
    float* meas_occ;
    float* meas_free;
    float* del_occ;
    float* del_free;
};

__device__ __forceinline__ void cell_xyz(int idx, int G, int* x, int* y, int* z) {
    // src/k3dom/kernel/mass_update.cu:92-94
    *x = idx % G;
    *y = (idx % (G * G)) / G;
    *z = idx / (G * G);
}

// Cell centre relative to the sensor in metres (mass_update.cu:92-99,
// measurement_grid.cu:77-84), with the reference's FP32 operation order.
__device__ __forceinline__ void cell_centre_rel(int idx, const DevParams& p, float sx, float sy,
                                                float sz, float* x, float* y, float* z) {
    int ix, iy, iz;
    cell_xyz(idx, p.G, &ix, &iy, &iz);
    float x_idx = __fadd_rn((float)ix, 0.5f);
    float y_idx = __fadd_rn((float)iy, 0.5f);
    float z_idx = __fadd_rn((float)iz, 0.5f);
    float hg = __fdiv_rn((float)p.G, 2.0f);
    float hz = __fdiv_rn((float)p.Gz, 2.0f);
    *x = __fsub_rn(__fmul_rn(__fsub_rn(x_idx, hg), p.res), sx);
    *y = __fsub_rn(__fmul_rn(__fsub_rn(y_idx, hg), p.res), sy);
    *z = __fsub_rn(__fmul_rn(__fsub_rn(z_idx, hz), p.res), sz);
}

// Saturating float -> int truncation with NaN -> 0, the behaviour of cvt.rzi.s32.f32.
__device__ __forceinline__ int f2i_trunc(float x) { return __float2int_rz(x); }

template <typename T>
__device__ __forceinline__ T clampv(T a, T lo, T hi) {
    // include/common/common.h:29-33: max(min(a, upper), lower)
    return max(min(a, hi), lo);
}

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

// Grid of a grid-stride kernel over n elements: at most kGridStrideCap blocks of kBlock.
constexpr int kGridStrideCap = 148 * 8;
inline int grid_for(long long n) {
    const int g = div_up(n, kBlock);
    return g < 1 ? 1 : (g > kGridStrideCap ? kGridStrideCap : g);
}

}  // namespace k3dom
