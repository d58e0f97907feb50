// cells.cu -- per-cell initialisation, the ego-motion map shift and the readback formats.
#include <cuda_runtime.h>

#include "common.cuh"
#include "internal.h"

namespace k3dom {

// initGridCellsKernel (src/common/kernel/init.cu:20-35): priors, empty ranges; every scene.
__global__ void k_cells_init(Batch bt, CellState cs, CellWork cw) {
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < bt.C; c += gridDim.x * blockDim.x) {
        const DevParams& p = bt.sc[scene_of(bt.off->cell, bt.S, c)].p;
        cs.free_m[c] = p.prior_free;
        cs.static_m[c] = p.prior_static;
        cs.dyn_m[c] = p.prior_dynamic;
        cs.occ_m[c] = p.prior_occ;
        cw.start[c] = -1;
        cw.end[c] = -1;
    }
}

void launch_cells_init(const Batch& bt, CellState cs, CellWork cw, cudaStream_t st) {
    ++g_launches;
    k_cells_init<<<grid_for(bt.C), kBlock, 0, st>>>(bt, cs, cw);
}

// The map part of DOM_c::updatePose (src/common/dom.cu:130-156): cells re-initialised to the
// priors (initGridCellsKernel), then moveMapKernel (ego_motion_compensation.cu:20-39)
// copies every GridCell whose source x+move lies inside the grid. Fields that
// initGridCellsKernel does not touch keep the value of the same index when the source is
// outside. The reference allocates and frees a copy per shift; here the two buffers are
// allocated once and flipped. born_m is not a GridCell field and is not moved.
__global__ void k_map_shift(DevParams p, CellState src, CellState dst, const int* __restrict__ s_start,
                            const int* __restrict__ s_end, int* __restrict__ d_start,
                            int* __restrict__ d_end, int mx, int my, int mz) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= p.C) return;
    int x, y, z;
    cell_xyz(c, p.G, &x, &y, &z);
    const int nx = x + mx, ny = y + my, nz = z + mz;
    const bool in = nx >= 0 && nx < p.G && ny >= 0 && ny < p.G && nz >= 0 && nz < p.Gz;
    const int q = in ? nx + p.G * ny + p.G * p.G * nz : c;
    if (in) {
        dst.free_m[c] = src.free_m[q];
        dst.static_m[c] = src.static_m[q];
        dst.dyn_m[c] = src.dyn_m[q];
        dst.occ_m[c] = src.occ_m[q];
        d_start[c] = s_start[q];
        d_end[c] = s_end[q];
    } else {
        dst.free_m[c] = p.prior_free;
        dst.static_m[c] = p.prior_static;
        dst.dyn_m[c] = p.prior_dynamic;
        dst.occ_m[c] = p.prior_occ;
        d_start[c] = -1;
        d_end[c] = -1;
    }
    dst.pers_m[c] = src.pers_m[q];
    dst.pred_m[c] = src.pred_m[q];
    dst.mvx[c] = src.mvx[q];
    dst.mvy[c] = src.mvy[q];
    dst.mvz[c] = src.mvz[q];
    dst.born_m[c] = src.born_m[c];
}

void launch_map_shift_full(const DevParams& p, CellState src, CellState dst, const int* s_start,
                           const int* s_end, int* d_start, int* d_end, int mx, int my, int mz,
                           cudaStream_t st) {
    ++g_launches;
    k_map_shift<<<div_up(p.C, kBlock), kBlock, 0, st>>>(p, src, dst, s_start, s_end, d_start, d_end,
                                                         mx, my, mz);
}


// ---------------------------------------------------------------- readback
struct CellView {
    float f, s, d, o, pers, pred, born, mvx, mvy, mvz, mu_A, mu_UA, w_A, w_UA, mocc, mfree, dlo, dlf;
    int start, end;
};

// Pointers are the scene's own ranges; range_base is the scene's first sorted particle, so the
// exported start/end are indices within the scene.
__device__ __forceinline__ void view_cell(const DevParams& p, int c, CellState cs, CellWork cw,
                                          const float* born_cum, int range_base, CellView& v) {
    v.f = cs.free_m[c]; v.s = cs.static_m[c]; v.d = cs.dyn_m[c]; v.o = cs.occ_m[c];
    v.pers = cs.pers_m[c]; v.pred = cs.pred_m[c]; v.born = cs.born_m[c];
    v.mvx = cs.mvx[c]; v.mvy = cs.mvy[c]; v.mvz = cs.mvz[c];
    v.start = cw.start[c]; v.end = cw.end[c];
    if (v.start >= 0) v.start -= range_base;
    if (v.end >= 0) v.end -= range_base;
    if (v.start >= 0) {
        // the factor the reweight applies: pers / pred (p_A = 0, so mu_A only multiplies 0)
        v.mu_UA = cw.factor[c];
        v.mu_A = v.mu_UA;
    } else {
        v.mu_A = v.mu_UA = 0.0f;
    }
    v.w_A = v.w_UA = 0.0f;
    if (born_cum) {
        // init_new_particles.cu:14-39,106-121 with p_A = 0
        const float mx = born_cum[p.C - 1];
        const float k = __fdiv_rn((float)p.B, mx);
        const int b1 = f2i_trunc(__fmul_rn(born_cum[c], k));
        const int b0 = c == 0 ? 0 : f2i_trunc(__fmul_rn(born_cum[c - 1], k));
        const int n = b0 <= b1 - 1 ? b1 - b0 : 0;
        const int nu_A = (int)roundf(__fmul_rn((float)n, p.p_A));
        const int nu_UA = n - nu_A;
        v.w_A = nu_A > 0 ? __fdiv_rn(__fmul_rn(p.p_A, v.born), (float)nu_A) : 0.0f;
        v.w_UA = nu_UA > 0 ? (float)((1.0 - (double)p.p_A) * (double)v.born / (double)nu_UA) : 0.0f;
    }
    v.mocc = cw.meas_occ ? cw.meas_occ[c] : 0.0f;
    v.mfree = cw.meas_free ? cw.meas_free[c] : 0.0f;
    v.dlo = cw.del_occ ? cw.del_occ[c] : 0.0f;
    v.dlf = cw.del_free ? cw.del_free[c] : 0.0f;
}

__device__ __forceinline__ float total_mass(const CellView& v) { return __fadd_rn(__fadd_rn(v.f, v.s), v.d); }

__global__ void k_export_field(DevParams p, int field, CellState cs, CellWork cw, const float* born_cum,
                               int range_base, float* dst) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= p.C) return;
    CellView v;
    view_cell(p, c, cs, cw, born_cum, range_base, v);
    float r = 0.0f;
    const float tm = total_mass(v);
    switch (field) {
        case 0: r = v.f; break;
        case 1: r = v.s; break;
        case 2: r = v.d; break;
        case 3: r = v.o; break;
        case 4: r = v.pers; break;
        case 5: r = v.pred; break;
        case 6: r = v.born; break;
        case 7: r = v.mvx; break;
        case 8: r = v.mvy; break;
        case 9: r = v.mvz; break;
        case 10: r = v.mu_A; break;
        case 11: r = v.mu_UA; break;
        case 12: r = v.w_A; break;
        case 13: r = v.w_UA; break;
        case 14: r = 1.0f; break;
        case 15: r = 0.0f; break;
        case 16: r = __fdiv_rn(__fadd_rn(v.s, v.d), tm); break;  // occ_mean, dom_types.h:48
        case 17: r = __fdiv_rn(v.d, tm); break;                   // dyn_mean, :49
        case 18: r = tm; break;                                     // total_mass, :47
        case 19: r = __fadd_rn(v.o, __fdiv_rn(__fsub_rn(__fsub_rn(1.0f, v.o), v.f), 2.0f)); break;  // :61
        case 20: {  // calcVar, :50-58
            if (tm == 0.0f) { r = 1e6f; break; }
            const float mm = fmaxf(fmaxf(v.f, v.s), v.d);
            const float mean = __fdiv_rn(mm, tm);
            r = __fdiv_rn(__fmul_rn(mean, __fsub_rn(1.0f, mean)), __fadd_rn(tm, 1.0f));
            break;
        }
        case 21: r = v.mocc; break;
        case 22: r = v.mfree; break;
        case 23: r = v.dlo; break;
        case 24: r = v.dlf; break;
        default: r = 0.0f;
    }
    dst[c] = r;
}

void launch_export_field(const DevParams& p, int field, CellState cs, CellWork cw, const float* born_cum,
                         int range_base, float* dst, cudaStream_t st) {
    ++g_launches;
    k_export_field<<<div_up(p.C, kBlock), kBlock, 0, st>>>(p, field, cs, cw, born_cum, range_base, dst);
}

// dom::GridCell, include/common/dom_types.h:12-45 (68 bytes).
struct GridCellAoS {
    int start_idx, end_idx;
    float mu_A, mu_UA, w_A, w_UA, mean_x_vel, mean_y_vel, mean_z_vel, likelihood, p_A;
    float free_mass, static_mass, dynamic_mass, occ_mass, pers_mass, pred_mass;
};
static_assert(sizeof(GridCellAoS) == 68, "GridCell layout");

__global__ void k_export_gridcell(DevParams p, CellState cs, CellWork cw, const float* born_cum,
                                  int range_base, GridCellAoS* dst) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= p.C) return;
    CellView v;
    view_cell(p, c, cs, cw, born_cum, range_base, v);
    GridCellAoS g;
    g.start_idx = v.start; g.end_idx = v.end;
    g.mu_A = v.mu_A; g.mu_UA = v.mu_UA; g.w_A = v.w_A; g.w_UA = v.w_UA;
    g.mean_x_vel = v.mvx; g.mean_y_vel = v.mvy; g.mean_z_vel = v.mvz;
    g.likelihood = 1.0f; g.p_A = 0.0f;
    g.free_mass = v.f; g.static_mass = v.s; g.dynamic_mass = v.d; g.occ_mass = v.o;
    g.pers_mass = v.pers; g.pred_mass = v.pred;
    dst[c] = g;
}

void launch_export_gridcell(const DevParams& p, CellState cs, CellWork cw, const float* born_cum,
                            int range_base, void* dst, cudaStream_t st) {
    ++g_launches;
    k_export_gridcell<<<div_up(p.C, kBlock), kBlock, 0, st>>>(p, cs, cw, born_cum, range_base,
                                                               reinterpret_cast<GridCellAoS*>(dst));
}

// /map_data point per cell (k3dom_node.cpp:161-184, DOM_c::indexToCoord* dom.h:70-81).
__global__ void k_export_mappoints(DevParams p, float cx, float cy, float cz, CellState cs, CellWork cw,
                                   float* dst) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= p.C) return;
    int ix, iy, iz;
    cell_xyz(c, p.G, &ix, &iy, &iz);
    const float hs = __fdiv_rn(p.size, 2.0f), hz = __fdiv_rn(p.size_z, 2.0f);
    float* o = dst + (long)c * 10;
    o[0] = __fadd_rn(__fsub_rn(__fmul_rn(__fadd_rn((float)ix, 0.5f), p.res), hs), cx);
    o[1] = __fadd_rn(__fsub_rn(__fmul_rn(__fadd_rn((float)iy, 0.5f), p.res), hs), cy);
    o[2] = __fadd_rn(__fsub_rn(__fmul_rn(__fadd_rn((float)iz, 0.5f), p.res), hz), cz);
    o[3] = __fmul_rn(cs.mvx[c], p.res);
    o[4] = __fmul_rn(cs.mvy[c], p.res);
    o[5] = __fmul_rn(cs.mvz[c], p.res);
    const float f = cs.free_m[c], s = cs.static_m[c], d = cs.dyn_m[c];
    const float tm = __fadd_rn(__fadd_rn(f, s), d);
    o[6] = __fdiv_rn(__fadd_rn(s, d), tm);
    o[7] = __fdiv_rn(d, tm);
    o[8] = tm;
    o[9] = 1.1f;
}

void launch_export_mappoints(const DevParams& p, float cx, float cy, float cz, CellState cs, CellWork cw,
                             float* dst, cudaStream_t st) {
    ++g_launches;
    k_export_mappoints<<<div_up(p.C, kBlock), kBlock, 0, st>>>(p, cx, cy, cz, cs, cw, dst);
}

}  // namespace k3dom
