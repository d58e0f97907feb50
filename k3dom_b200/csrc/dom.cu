// dom.cu -- host orchestration behind the C ABI: the B200 counterpart of dom::DOM_c and the
// two dom::DOM variants (src/common/dom.cu, src/k3dom/dom.cu, src/dsphdmib/dom.cu).
//
// Differences in structure from the reference, by design:
//  * every buffer is allocated once at creation (the reference allocates measurement arrays,
//    Thrust temporaries and a map copy on every frame);
//  * no host synchronisation inside a frame (the reference reads scalars back at
//    init_new_particles.cu:49, src/common/dom.cu:275 and resampling.cu:58), so the
//    steady-state frame can be captured in a CUDA graph and replayed;
//  * particles are double-buffered by role (current / sorted / birth) instead of the deep
//    copy particle_array = particle_array_next (src/k3dom/dom.cu:43);
//  * resampling draws are generated and sorted on a second stream while the evidence
//    kernel runs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/k3dom_b200.h"
#include "common.cuh"
#include "internal.h"

using namespace k3dom;

namespace k3dom {
cudaError_t exact_scan_float2(const float* a, long na, const float* b, long nb, float* out, void* scratch,
                              cudaStream_t st);
}

#define CK(x)                                  \
    do {                                       \
        cudaError_t e_ = (x);                  \
        if (e_ != cudaSuccess) return fail(e_); \
    } while (0)

struct k3dom_handle {
    int device = 0;
    int num_sms = 148;
    k3dom_variant variant = K3DOM_VARIANT_K3DOM;
    k3dom_params params{};
    DevParams dp{};
    EvidenceConfig ec{};
    cudaStream_t st = nullptr, st2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaEvent_t ev_t[8] = {};
    bool timing = false;
    k3dom_stage_times times{};

    FrameParams* fp_dev = nullptr;
    FrameParams* fp_host = nullptr;  // pinned
    DevStatus* status = nullptr;

    Particles A{}, S{}, Bp{};
    uint32_t *sorted_keys = nullptr, *perm = nullptr, *alt_k = nullptr, *alt_v = nullptr;
    uint32_t *hist = nullptr, *scan_tmp = nullptr;
    long hist_words = 0, scan_tmp_words = 0;
    CellState cs[2]{};  // cs[0] live, cs[1] spare for the map shift
    int *start2 = nullptr, *end2 = nullptr;
    CellWork cw{};
    float *born_cum = nullptr, *joint_cum = nullptr, *joint_max = nullptr;
    void* exact_scratch = nullptr;
    uint32_t *draw_keys = nullptr, *draw_sorted = nullptr, *draw_alt = nullptr;
    uint32_t *hist_draw = nullptr, *scan_tmp_draw = nullptr;
    cudaEvent_t ev_staged = nullptr;  // host staging (frame scalars, points) consumed
    int* ancestors = nullptr;
    float *pts = nullptr;       // device x | y | z (3 * max_points)
    float* pts_pinned = nullptr;
    RayBuffers rb{};
    void* export_buf = nullptr;
    size_t export_bytes = 0;
    std::vector<void*> allocs;

    // DOM_c host state (include/common/dom.h:135-147)
    bool first_pose_received = false;
    float sensor_pos[3] = {0, 0, 0}, center_pos[3] = {0, 0, 0};
    float updated_time = -1.0f;
    int iteration = 0;
    uint32_t frame = 0;
    bool shift_pending = false;
    int pending_shift[3] = {0, 0, 0};
    bool births_done = false;
    int launches_per_frame = 0;
    bool initialized = false;

    // graph of the steady-state frame
    bool graph_mode = true;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int graph_npts = -1;

    cudaError_t last_error = cudaSuccess;
    k3dom_status fail(cudaError_t e) {
        last_error = e;
        return e == cudaErrorMemoryAllocation ? K3DOM_ERR_OUT_OF_MEMORY : K3DOM_ERR_CUDA;
    }

    template <typename T>
    cudaError_t alloc(T** p, size_t count, bool zero = true) {
        *p = nullptr;
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
        if (e != cudaSuccess) return e;
        allocs.push_back((void*)*p);
        if (zero) e = cudaMemset(*p, 0, count * sizeof(T));
        return e;
    }
    cudaError_t alloc_particles(Particles* q, int n) {
        cudaError_t e;
        if ((e = alloc(&q->px, n)) || (e = alloc(&q->py, n)) || (e = alloc(&q->pz, n)) || (e = alloc(&q->vx, n)) ||
            (e = alloc(&q->vy, n)) || (e = alloc(&q->vz, n)) || (e = alloc(&q->w, n)) || (e = alloc(&q->cell, n)) ||
            (e = alloc(&q->assoc, n)))
            return e;
        return cudaSuccess;
    }
    cudaError_t alloc_cells(CellState* c, int n) {
        cudaError_t e;
        if ((e = alloc(&c->free_m, n)) || (e = alloc(&c->static_m, n)) || (e = alloc(&c->dyn_m, n)) ||
            (e = alloc(&c->occ_m, n)) || (e = alloc(&c->pers_m, n)) || (e = alloc(&c->pred_m, n)) ||
            (e = alloc(&c->born_m, n)) || (e = alloc(&c->mvx, n)) || (e = alloc(&c->mvy, n)) ||
            (e = alloc(&c->mvz, n)))
            return e;
        return cudaSuccess;
    }
    void release() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        graph_exec = nullptr;
        graph = nullptr;
        for (void* p : allocs) cudaFree(p);
        allocs.clear();
        if (fp_host) cudaFreeHost(fp_host);
        if (pts_pinned) cudaFreeHost(pts_pinned);
        if (export_buf) cudaFree(export_buf);
        for (auto& e : ev_t)
            if (e) cudaEventDestroy(e);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (ev_staged) cudaEventDestroy(ev_staged);
        if (st) cudaStreamDestroy(st);
        if (st2) cudaStreamDestroy(st2);
    }
    CellState cells() const { return cs[0]; }
};

namespace {

int key_bits_for(long n) {
    int b = 1;
    while (b < 31 && (1L << b) < n) ++b;
    return b;
}

k3dom_status validate(const k3dom_params* p, k3dom_variant v) {
    if (!p) return K3DOM_ERR_INVALID_ARGUMENT;
    if (v != K3DOM_VARIANT_K3DOM && v != K3DOM_VARIANT_DSPHDMIB) return K3DOM_ERR_INVALID_ARGUMENT;
    if (!(p->resolution > 0.0f) || !std::isfinite(p->resolution)) return K3DOM_ERR_INVALID_ARGUMENT;
    if (!(p->size > 0.0f) || !(p->size_z > 0.0f)) return K3DOM_ERR_INVALID_ARGUMENT;
    const int G = static_cast<int>(p->size / p->resolution), Gz = static_cast<int>(p->size_z / p->resolution);
    if (G < 1 || Gz < 1) return K3DOM_ERR_INVALID_ARGUMENT;
    if ((double)G * G * Gz > 2147483647.0 / 2) return K3DOM_ERR_CAPACITY;
    if (p->particle_count < 1 || p->new_born_particle_count < 1) return K3DOM_ERR_INVALID_ARGUMENT;
    if ((long)p->particle_count + p->new_born_particle_count > (1L << 30)) return K3DOM_ERR_CAPACITY;
    if (v == K3DOM_VARIANT_K3DOM && (!(p->ls > 0.0f) || !(p->sigma >= 0.0f) || !(p->mass_scale != 0.0f)))
        return K3DOM_ERR_INVALID_ARGUMENT;
    if (v == K3DOM_VARIANT_DSPHDMIB && (!(p->max_range > 0.0f) || !(p->meas_occ_stddev > 0.0f)))
        return K3DOM_ERR_INVALID_ARGUMENT;
    return K3DOM_OK;
}

cudaError_t alloc_ray_buffers(k3dom_handle* h, int max_points) {
    RayBuffers& rb = h->rb;
    rb.max_points = max_points;
    rb.tx = h->ec.tile_x;
    rb.ty = h->ec.tile_y;
    rb.tz = h->ec.tile_z;
    rb.ntx = (h->dp.G + rb.tx - 1) / rb.tx;
    rb.nty = (h->dp.G + rb.ty - 1) / rb.ty;
    rb.ntz = (h->dp.Gz + rb.tz - 1) / rb.tz;
    rb.tiles = rb.ntx * rb.nty * rb.ntz;
    long cap = ray_entries_bound(h->dp, h->ec, max_points);
    cap = std::max(cap, 4096L);
    rb.capacity = cap;
    cudaError_t e;
    if ((e = h->alloc(&rb.ray_a, max_points)) || (e = h->alloc(&rb.ray_b, max_points)) ||
        (e = h->alloc(&rb.ray_c, max_points)) ||
        (e = h->alloc(&rb.counts, max_points)) || (e = h->alloc(&rb.offsets, max_points)) ||
        (e = h->alloc(&rb.ekeys, cap, false)) || (e = h->alloc(&rb.evals, cap, false)) ||
        (e = h->alloc(&rb.ekeys2, cap, false)) || (e = h->alloc(&rb.evals2, cap, false)) ||
        (e = h->alloc(&rb.tile_start, rb.tiles + 1)) || (e = h->alloc(&rb.tile_items, rb.tiles)) ||
        (e = h->alloc(&rb.item_off, rb.tiles + 1)) || (e = h->alloc(&rb.tile_done, rb.tiles)) ||
        (e = h->alloc(&rb.acc, 2 * (size_t)h->dp.C)) || (e = h->alloc(&rb.total, 4)) ||
        (e = h->alloc(&rb.ktab, kKernelTableSize)))
        return e;
    {
        std::vector<float4> tab(kKernelTableSize);
        build_kernel_table(h->dp.sigma, tab.data());
        if ((e = cudaMemcpy(rb.ktab, tab.data(), sizeof(float4) * tab.size(), cudaMemcpyHostToDevice))) return e;
    }
    int bits = 1;
    while ((1 << bits) < rb.tiles + 1) ++bits;
    int pb[4];
    if (radix_plan(bits, pb) > 1) {
        if ((e = h->alloc(&rb.ekeys_alt, cap, false)) || (e = h->alloc(&rb.evals_alt, cap, false))) return e;
    } else {
        rb.ekeys_alt = rb.ekeys;
        rb.evals_alt = rb.evals;
    }
    const long items_max = rb.tiles + cap / 1024 + 2;
    const long tile_cells = (long)rb.tx * rb.ty * rb.tz;
    if (h->variant == K3DOM_VARIANT_DSPHDMIB) {
        rb.ds_count_capacity = items_max * tile_cells;
        if ((e = h->alloc(&rb.ds_counts, rb.ds_count_capacity))) return e;
    } else {
        rb.ds_count_capacity = 0;
    }
    // shared sort/scan scratch sized for the largest user
    const long hw = std::max({radix_hist_words(h->dp.P, 11), radix_hist_words(cap, 11), 1L});
    if (hw > h->hist_words) {
        if ((e = h->alloc(&h->hist, hw))) return e;
        h->hist_words = hw;
    }
    const long sw = scan_u32_tiles(std::max({hw, (long)max_points, (long)rb.tiles + 1})) + 16;
    if (sw > h->scan_tmp_words) {
        if ((e = h->alloc(&h->scan_tmp, sw))) return e;
        h->scan_tmp_words = sw;
    }
    rb.hist = h->hist;
    rb.scan_tmp = h->scan_tmp;
    if ((e = h->alloc(&h->pts, 3 * (size_t)max_points))) return e;
    if (h->pts_pinned) cudaFreeHost(h->pts_pinned);
    if ((e = cudaMallocHost((void**)&h->pts_pinned, 3 * (size_t)max_points * sizeof(float)))) return e;
    return cudaSuccess;
}

void choose_tiles(k3dom_handle* h) {
    // 16x16x8-cell tiles for large grids, 8x8x4 for small ones
    if ((long)h->dp.C >= (1L << 20) && h->dp.Gz >= 8) {
        h->ec.tile_x = 16; h->ec.tile_y = 16; h->ec.tile_z = 8;
    } else {
        h->ec.tile_x = 8; h->ec.tile_y = 8; h->ec.tile_z = 4;
    }
    h->ec.chunk = 1024;
}

}  // namespace

// ===================================================================== frame pieces
namespace {

k3dom_status set_frame_params(k3dom_handle* h, float dt, int n_points) {
    // the pinned staging (frame scalars and points) may still be read by an earlier copy
    cudaError_t e = cudaEventSynchronize(h->ev_staged);
    if (e != cudaSuccess) return h->fail(e);
    FrameParams& f = *h->fp_host;
    f.dt = dt;
    f.sensor_x = h->sensor_pos[0] - h->center_pos[0];
    f.sensor_y = h->sensor_pos[1] - h->center_pos[1];
    f.sensor_z = h->sensor_pos[2] - h->center_pos[2];
    f.n_points = n_points;
    f.frame = h->frame;
    f.shift_x = h->pending_shift[0];
    f.shift_y = h->pending_shift[1];
    f.shift_z = h->pending_shift[2];
    f.shift_pending = h->shift_pending ? 1 : 0;
    f.seed = h->params.seed;
    e = cudaMemcpyAsync(h->fp_dev, h->fp_host, sizeof(FrameParams), cudaMemcpyHostToDevice, h->st);
    if (e != cudaSuccess) return h->fail(e);
    e = cudaEventRecord(h->ev_staged, h->st);
    return e == cudaSuccess ? K3DOM_OK : h->fail(e);
}

k3dom_status grow_points(k3dom_handle* h, int n) {
    if (n <= h->rb.max_points) return K3DOM_OK;
    // capacity grows (allocation happens only here, outside the steady state)
    cudaError_t e = cudaStreamSynchronize(h->st);
    if (e != cudaSuccess) return h->fail(e);
    auto drop = [&](void* p) {
        if (!p) return;
        auto it = std::find(h->allocs.begin(), h->allocs.end(), p);
        if (it != h->allocs.end()) { cudaFree(p); h->allocs.erase(it); }
    };
    RayBuffers& rb = h->rb;
    for (void* p : {(void*)rb.ray_a, (void*)rb.ray_b, (void*)rb.ray_c, (void*)rb.counts, (void*)rb.offsets, (void*)rb.ekeys,
                    (void*)rb.evals, (void*)rb.ekeys2, (void*)rb.evals2, (void*)rb.tile_start, (void*)rb.tile_items,
                    (void*)rb.item_off, (void*)rb.tile_done, (void*)rb.acc, (void*)rb.total, (void*)rb.ds_counts,
                    (void*)rb.ktab,
                    (void*)h->pts})
        drop(p);
    if (rb.ekeys_alt != rb.ekeys) { drop(rb.ekeys_alt); drop(rb.evals_alt); }
    int np = std::max(n, (int)(rb.max_points * 1.25));
    e = alloc_ray_buffers(h, np);
    if (e != cudaSuccess) return h->fail(e);
    if (h->graph_exec) { cudaGraphExecDestroy(h->graph_exec); h->graph_exec = nullptr; }
    if (h->graph) { cudaGraphDestroy(h->graph); h->graph = nullptr; }
    h->params.max_points = np;
    return K3DOM_OK;
}

// Points -> device SoA. Host input is staged through pinned memory.
k3dom_status upload_points(k3dom_handle* h, const float* xs, const float* ys, const float* zs, int n, k3dom_mem mem) {
    if (n < 0) return K3DOM_ERR_INVALID_ARGUMENT;
    if (n > 0 && !xs) return K3DOM_ERR_INVALID_ARGUMENT;
    k3dom_status s = grow_points(h, n);
    if (s != K3DOM_OK) return s;
    const int M = h->rb.max_points;
    float* dx = h->pts;
    float* dy = h->pts + M;
    float* dz = h->pts + 2 * (size_t)M;
    if (n == 0) return K3DOM_OK;
    const bool interleaved = (ys == nullptr || zs == nullptr);
    cudaError_t e;
    if (mem == K3DOM_MEM_HOST) {
        // stage in pinned memory (previous frame's copies completed: set_frame_params synced)
        float* hx = h->pts_pinned;
        float* hy = hx + M;
        float* hz = hx + 2 * (size_t)M;
        if (interleaved) {
            for (int i = 0; i < n; ++i) {
                hx[i] = xs[3 * i];
                hy[i] = xs[3 * i + 1];
                hz[i] = xs[3 * i + 2];
            }
        } else {
            std::memcpy(hx, xs, n * sizeof(float));
            std::memcpy(hy, ys, n * sizeof(float));
            std::memcpy(hz, zs, n * sizeof(float));
        }
        if ((e = cudaMemcpyAsync(dx, hx, n * sizeof(float), cudaMemcpyHostToDevice, h->st)) ||
            (e = cudaMemcpyAsync(dy, hy, n * sizeof(float), cudaMemcpyHostToDevice, h->st)) ||
            (e = cudaMemcpyAsync(dz, hz, n * sizeof(float), cudaMemcpyHostToDevice, h->st)))
            return h->fail(e);
        if ((e = cudaEventRecord(h->ev_staged, h->st))) return h->fail(e);
    } else {
        if (interleaved) {
            if ((e = cudaMemcpy2DAsync(dx, sizeof(float), xs, 3 * sizeof(float), sizeof(float), n,
                                       cudaMemcpyDeviceToDevice, h->st)) ||
                (e = cudaMemcpy2DAsync(dy, sizeof(float), xs + 1, 3 * sizeof(float), sizeof(float), n,
                                       cudaMemcpyDeviceToDevice, h->st)) ||
                (e = cudaMemcpy2DAsync(dz, sizeof(float), xs + 2, 3 * sizeof(float), sizeof(float), n,
                                       cudaMemcpyDeviceToDevice, h->st)))
                return h->fail(e);
        } else {
            if ((e = cudaMemcpyAsync(dx, xs, n * sizeof(float), cudaMemcpyDeviceToDevice, h->st)) ||
                (e = cudaMemcpyAsync(dy, ys, n * sizeof(float), cudaMemcpyDeviceToDevice, h->st)) ||
                (e = cudaMemcpyAsync(dz, zs, n * sizeof(float), cudaMemcpyDeviceToDevice, h->st)))
                return h->fail(e);
        }
    }
    return K3DOM_OK;
}

bool has_nonfinite_host(const float* xs, const float* ys, const float* zs, int n) {
    const bool inter = (ys == nullptr || zs == nullptr);
    const long m = inter ? 3L * n : n;
    for (long i = 0; i < m; ++i)
        if (!std::isfinite(xs[i])) return true;
    if (!inter)
        for (int i = 0; i < n; ++i)
            if (!std::isfinite(ys[i]) || !std::isfinite(zs[i])) return true;
    return false;
}

void rec(k3dom_handle* h, int i) {
    if (h->timing) cudaEventRecord(h->ev_t[i], h->st);
}

// --- enqueue helpers (no synchronisation) ---
cudaError_t enq_predict(k3dom_handle* h) {
    launch_predict(h->dp, h->fp_dev, h->A, h->st);
    return cudaGetLastError();
}

cudaError_t enq_assign(k3dom_handle* h) {
    const DevParams& p = h->dp;
    cudaError_t e = radix_sort_pairs(reinterpret_cast<const uint32_t*>(h->A.cell), nullptr, h->sorted_keys, h->perm,
                                     h->alt_k, h->alt_v, p.P, key_bits_for(p.C), h->hist, h->scan_tmp, h->st);
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(h->cw.start, 0xFF, sizeof(int) * (size_t)p.C, h->st))) return e;
    if ((e = cudaMemsetAsync(h->cw.end, 0xFF, sizeof(int) * (size_t)p.C, h->st))) return e;
    launch_gather_segsum(p, h->A, h->S, h->sorted_keys, h->perm, h->cw, h->st);
    return cudaGetLastError();
}

cudaError_t enq_occupancy(k3dom_handle* h, bool first_frame) {
    const DevParams& p = h->dp;
    const int M = h->rb.max_points;
    const bool ds = h->variant == K3DOM_VARIANT_DSPHDMIB;
    cudaError_t e = build_ray_lists(p, h->fp_dev, h->pts, h->pts + M, h->pts + 2 * (size_t)M, h->rb, ds,
                                    h->status, h->st);
    if (e != cudaSuccess) return e;
    rec(h, 7);
    if (ds)
        e = launch_ds_evidence(p, h->fp_dev, h->rb, h->cells(), h->cw, first_frame, h->status, h->num_sms, h->st);
    else
        e = launch_k3dom_evidence(p, h->fp_dev, h->rb, h->cells(), h->cw, first_frame, h->status, h->num_sms, h->st);
    return e;
}

cudaError_t enq_persistent(k3dom_handle* h) {
    launch_reweight(h->dp, h->S, h->sorted_keys, h->cw, h->st);
    return cudaGetLastError();
}

cudaError_t enq_births(k3dom_handle* h) {
    const DevParams& p = h->dp;
    cudaError_t e = exact_scan_float(h->cells().born_m, h->born_cum, p.C, h->exact_scratch, h->st);
    if (e != cudaSuccess) return e;
    launch_births(p, h->fp_dev, h->cells().born_m, h->born_cum, h->Bp, h->st);
    return cudaGetLastError();
}

cudaError_t enq_draws(k3dom_handle* h, cudaStream_t s) {
    const DevParams& p = h->dp;
    launch_draw_keys(p, h->fp_dev, h->draw_keys, s);
    return radix_sort_pairs(h->draw_keys, nullptr, h->draw_sorted, nullptr, h->draw_alt, nullptr, p.P, 24,
                            h->hist_draw, h->scan_tmp_draw, s);
}

cudaError_t enq_resample(k3dom_handle* h, bool draws_ready) {
    const DevParams& p = h->dp;
    cudaError_t e;
    if (!draws_ready) {
        if ((e = enq_draws(h, h->st))) return e;
    }
    launch_joint_prepare(p, h->S, h->Bp, nullptr, h->st);
    if ((e = exact_scan_float2(h->S.w, p.P, h->Bp.w, p.B, h->joint_cum, h->exact_scratch, h->st))) return e;
    launch_resample(p, h->joint_cum, h->draw_sorted, h->S, h->sorted_keys, h->Bp, h->A, h->ancestors, h->joint_max,
                    h->st);
    return cudaGetLastError();
}

cudaError_t enq_init_particles(k3dom_handle* h) {
    const DevParams& p = h->dp;
    cudaError_t e = exact_scan_float(h->cells().born_m, h->born_cum, p.C, h->exact_scratch, h->st);
    if (e != cudaSuccess) return e;
    launch_init_particles(p, h->fp_dev, h->born_cum, h->A, h->st);
    return cudaGetLastError();
}

// The steady-state frame (DOM::updateGrid's branch for updated_time > 0).
cudaError_t enq_frame(k3dom_handle* h) {
    cudaError_t e;
    const long l0 = g_launches;
    // resampling draws depend only on (seed, frame): produce them beside the frame
    if ((e = cudaEventRecord(h->ev_fork, h->st))) return e;
    if ((e = cudaStreamWaitEvent(h->st2, h->ev_fork, 0))) return e;
    if ((e = enq_draws(h, h->st2))) return e;
    if ((e = cudaEventRecord(h->ev_join, h->st2))) return e;
    rec(h, 0);
    if ((e = enq_predict(h))) return e;
    rec(h, 1);
    if ((e = enq_assign(h))) return e;
    rec(h, 2);
    if ((e = enq_occupancy(h, false))) return e;
    rec(h, 3);
    if ((e = enq_persistent(h))) return e;
    rec(h, 4);
    if ((e = enq_births(h))) return e;
    rec(h, 5);
    if ((e = cudaStreamWaitEvent(h->st, h->ev_join, 0))) return e;
    if ((e = enq_resample(h, true))) return e;
    rec(h, 6);
    h->launches_per_frame = (int)(g_launches - l0);
    return cudaSuccess;
}

void read_times(k3dom_handle* h) {
    if (!h->timing) return;
    float t[7] = {0};
    for (int i = 0; i < 6; ++i) cudaEventElapsedTime(&t[i], h->ev_t[i], h->ev_t[i + 1]);
    h->times.predict_ms = t[0];
    h->times.assign_ms = t[1];
    h->times.occupancy_ms = t[2];
    h->times.persistent_ms = t[3];
    h->times.births_ms = t[4];
    h->times.resample_ms = t[5];
    cudaEventElapsedTime(&h->times.total_ms, h->ev_t[0], h->ev_t[6]);
    cudaEventElapsedTime(&h->times.binning_ms, h->ev_t[2], h->ev_t[7]);
    cudaEventElapsedTime(&h->times.evidence_ms, h->ev_t[7], h->ev_t[3]);
}

}  // namespace

// ===================================================================== C ABI
extern "C" {

static cudaError_t copy_cells_back(k3dom_handle* h);

const char* k3dom_status_string(k3dom_status s) {
    switch (s) {
        case K3DOM_OK: return "ok";
        case K3DOM_ERR_INVALID_ARGUMENT: return "invalid argument";
        case K3DOM_ERR_CUDA: return "CUDA error";
        case K3DOM_ERR_OUT_OF_MEMORY: return "out of device memory";
        case K3DOM_ERR_CAPACITY: return "capacity exceeded";
        case K3DOM_ERR_NOT_READY: return "not ready (call order)";
        case K3DOM_ERR_TIMEOUT: return "device wait timed out";
        case K3DOM_ERR_IO: return "file could not be read";
        case K3DOM_ERR_INVALID_INPUT: return "non-finite input";
        case K3DOM_ERR_NO_DEVICE: return "no CUDA device";
    }
    return "unknown status";
}

int32_t k3dom_abi_version(void) { return K3DOM_B200_ABI_VERSION; }

k3dom_status k3dom_create(const k3dom_params* params, k3dom_variant variant, int device, k3dom_handle** out) {
    if (!out) return K3DOM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    k3dom_status s = validate(params, variant);
    if (s != K3DOM_OK) return s;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return K3DOM_ERR_NO_DEVICE;
    if (device < 0 || device >= ndev) return K3DOM_ERR_INVALID_ARGUMENT;
    k3dom_handle* h = new (std::nothrow) k3dom_handle();
    if (!h) return K3DOM_ERR_OUT_OF_MEMORY;
    h->device = device;
    h->variant = variant;
    h->params = *params;
    if (h->params.max_points <= 0) h->params.max_points = 131072;
    auto bail = [&](cudaError_t e) {
        k3dom_status r = h->fail(e);
        h->release();
        delete h;
        return r;
    };
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return bail(e);
    cudaDeviceProp prop;
    if ((e = cudaGetDeviceProperties(&prop, device))) return bail(e);
    h->num_sms = prop.multiProcessorCount;
    if ((e = sort_init()) || (e = evidence_init())) return bail(e);

    DevParams& d = h->dp;
    const k3dom_params& p = h->params;
    d.G = static_cast<int>(p.size / p.resolution);          // src/common/dom.cu:30
    d.Gz = static_cast<int>(p.size_z / p.resolution);
    d.C = d.G * d.G * d.Gz;
    d.P = p.particle_count;
    d.B = p.new_born_particle_count;
    d.res = p.resolution;
    d.size = p.size;
    d.size_z = p.size_z;
    d.mass_scale = p.mass_scale;
    d.p_S = p.persistence_prob;
    d.noise_pos = p.stddev_process_noise_position;
    d.noise_vel = p.stddev_process_noise_velocity;
    d.p_B = p.birth_prob;
    d.stddev_vel = p.stddev_velocity;
    d.init_max_vel = p.init_max_velocity;
    d.min_vel = p.particle_min_vel;
    d.prior_free = p.prior_free;
    d.prior_static = p.prior_static;
    d.prior_dynamic = p.prior_dynamic;
    d.prior_occ = p.prior_occ;
    d.sigma = p.sigma;
    d.ls = p.ls;
    d.gamma = p.gamma;
    d.max_range = p.max_range;
    d.meas_occ_stddev = p.meas_occ_stddev;
    d.window_radius = p.resolution * 0.866f;  // src/dsphdmib/dom.cu:22
    d.p_A = 0.0f;
    d.likelihood = 1.0f;
    d.seed = p.seed;
    d.variant = (int)variant;
    choose_tiles(h);

    if ((e = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking))) return bail(e);
    if ((e = cudaStreamCreateWithFlags(&h->st2, cudaStreamNonBlocking))) return bail(e);
    if ((e = cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming))) return bail(e);
    if ((e = cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming))) return bail(e);
    if ((e = cudaEventCreateWithFlags(&h->ev_staged, cudaEventDisableTiming))) return bail(e);
    if ((e = cudaEventRecord(h->ev_staged, h->st))) return bail(e);
    for (auto& ev : h->ev_t)
        if ((e = cudaEventCreate(&ev))) return bail(e);
    if ((e = cudaMallocHost((void**)&h->fp_host, sizeof(FrameParams)))) return bail(e);
    std::memset(h->fp_host, 0, sizeof(FrameParams));
    if ((e = h->alloc(&h->fp_dev, 1)) || (e = h->alloc(&h->status, 1))) return bail(e);
    if ((e = h->alloc_particles(&h->A, d.P)) || (e = h->alloc_particles(&h->S, d.P)) ||
        (e = h->alloc_particles(&h->Bp, d.B)))
        return bail(e);
    if ((e = h->alloc(&h->sorted_keys, d.P)) || (e = h->alloc(&h->perm, d.P)) || (e = h->alloc(&h->alt_k, d.P)) ||
        (e = h->alloc(&h->alt_v, d.P)))
        return bail(e);
    if ((e = h->alloc_cells(&h->cs[0], d.C)) || (e = h->alloc_cells(&h->cs[1], d.C))) return bail(e);
    CellWork& cw = h->cw;
    if ((e = h->alloc(&cw.start, d.C)) || (e = h->alloc(&cw.end, d.C)) || (e = h->alloc(&h->start2, d.C)) ||
        (e = h->alloc(&h->end2, d.C)) || (e = h->alloc(&cw.sum_w, d.C)) || (e = h->alloc(&cw.sum_wvx, d.C)) ||
        (e = h->alloc(&cw.sum_wvy, d.C)) || (e = h->alloc(&cw.sum_wvz, d.C)) || (e = h->alloc(&cw.factor, d.C)) ||
        (e = h->alloc(&cw.divisor, d.C)) || (e = h->alloc(&cw.meas_occ, d.C)) || (e = h->alloc(&cw.meas_free, d.C)) ||
        (e = h->alloc(&cw.del_occ, d.C)) || (e = h->alloc(&cw.del_free, d.C)))
        return bail(e);
    if ((e = h->alloc(&h->born_cum, d.C)) || (e = h->alloc(&h->joint_cum, (size_t)d.P + d.B)) ||
        (e = h->alloc(&h->joint_max, 1)) || (e = h->alloc(&h->ancestors, d.P)))
        return bail(e);
    {
        const size_t sb = std::max(exact_scan_scratch_bytes((long)d.P + d.B), exact_scan_scratch_bytes(d.C));
        unsigned char* es = nullptr;
        if ((e = h->alloc(&es, sb))) return bail(e);
        h->exact_scratch = es;
    }
    if ((e = h->alloc(&h->draw_keys, d.P)) || (e = h->alloc(&h->draw_sorted, d.P)) ||
        (e = h->alloc(&h->draw_alt, d.P)))
        return bail(e);
    // separate sort scratch for the draw sort (it runs concurrently on the second stream)
    {
        const long hw = radix_hist_words(d.P, 8);
        if ((e = h->alloc(&h->hist_draw, hw))) return bail(e);
        if ((e = h->alloc(&h->scan_tmp_draw, scan_u32_tiles(hw) + 16))) return bail(e);
    }
    if ((e = alloc_ray_buffers(h, h->params.max_points))) return bail(e);
    // DOM_c::initialize (src/common/dom.cu:90-109): cells to priors
    launch_cells_init(d, h->cs[0], h->cw, h->st);
    launch_cells_init(d, h->cs[1], h->cw, h->st);
    if ((e = cudaGetLastError()) || (e = cudaStreamSynchronize(h->st))) return bail(e);
    *out = h;
    return K3DOM_OK;
}

k3dom_status k3dom_destroy(k3dom_handle* h) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->st);
    cudaStreamSynchronize(h->st2);
    h->release();
    delete h;
    return K3DOM_OK;
}

k3dom_status k3dom_update_pose(k3dom_handle* h, float x, float y, float z) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    const k3dom_params& p = h->params;
    h->sensor_pos[0] = x;
    h->sensor_pos[1] = y;
    h->sensor_pos[2] = z;
    if (!h->first_pose_received) {
        h->first_pose_received = true;
        h->center_pos[0] = x - p.sensor_off_x;
        h->center_pos[1] = y - p.sensor_off_y;
        h->center_pos[2] = z - p.sensor_off_z;
        return K3DOM_OK;
    }
    const int mx = static_cast<int>((x - h->center_pos[0] - p.sensor_off_x) / p.resolution);
    const int my = static_cast<int>((y - h->center_pos[1] - p.sensor_off_y) / p.resolution);
    const int mz = static_cast<int>((z - h->center_pos[2] - p.sensor_off_z) / p.resolution);
    if (std::abs(mx) >= p.map_shift_thresh || std::abs(my) >= p.map_shift_thresh ||
        std::abs(mz) >= p.map_shift_thresh) {
        cudaError_t e;
        if (h->shift_pending) {
            // a second shift before any prediction: apply the first to the particles now so
            // each subtraction rounds exactly as moveParticlesKernel's would
            launch_shift_particles(h->dp, h->A, h->pending_shift[0], h->pending_shift[1], h->pending_shift[2], h->st);
        }
        // shift into the spare buffers, then copy back so every captured pointer stays valid
        launch_map_shift_full(h->dp, h->cs[0], h->cs[1], h->cw.start, h->cw.end, h->start2, h->end2, mx, my, mz,
                              h->st);
        if ((e = copy_cells_back(h))) return h->fail(e);
        h->shift_pending = true;
        h->pending_shift[0] = mx;
        h->pending_shift[1] = my;
        h->pending_shift[2] = mz;
        if ((e = cudaGetLastError())) return h->fail(e);
        h->center_pos[0] += mx * p.resolution;
        h->center_pos[1] += my * p.resolution;
        h->center_pos[2] += mz * p.resolution;
    }
    return K3DOM_OK;
}

static cudaError_t copy_cells_back(k3dom_handle* h) {
    const size_t b = sizeof(float) * (size_t)h->dp.C;
    const CellState& s = h->cs[1];
    const CellState& d = h->cs[0];
    const float* src[] = {s.free_m, s.static_m, s.dyn_m, s.occ_m, s.pers_m, s.pred_m, s.born_m, s.mvx, s.mvy, s.mvz};
    float* dst[] = {d.free_m, d.static_m, d.dyn_m, d.occ_m, d.pers_m, d.pred_m, d.born_m, d.mvx, d.mvy, d.mvz};
    cudaError_t e;
    for (int i = 0; i < 10; ++i)
        if ((e = cudaMemcpyAsync(dst[i], src[i], b, cudaMemcpyDeviceToDevice, h->st))) return e;
    if ((e = cudaMemcpyAsync(h->cw.start, h->start2, sizeof(int) * (size_t)h->dp.C, cudaMemcpyDeviceToDevice, h->st)))
        return e;
    return cudaMemcpyAsync(h->cw.end, h->end2, sizeof(int) * (size_t)h->dp.C, cudaMemcpyDeviceToDevice, h->st);
}

static k3dom_status finish_sync(k3dom_handle* h) {
    cudaError_t e = cudaStreamSynchronize(h->st);
    if (e != cudaSuccess) return h->fail(e);
    if (h->status) {
        DevStatus st;
        e = cudaMemcpy(&st, h->status, sizeof(st), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return h->fail(e);
        if (st.overflow) return K3DOM_ERR_CAPACITY;
    }
    return K3DOM_OK;
}

static k3dom_status update_grid_impl(k3dom_handle* h, float t, const float* xs, const float* ys, const float* zs,
                                     int32_t n, k3dom_mem mem, bool sync) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    if (n < 0 || (n > 0 && !xs)) return K3DOM_ERR_INVALID_ARGUMENT;
    if (mem == K3DOM_MEM_HOST && n > 0 && has_nonfinite_host(xs, ys, zs, n)) return K3DOM_ERR_INVALID_INPUT;
    cudaSetDevice(h->device);
    const bool steady = h->updated_time > 0.0f;  // src/k3dom/dom.cu:32
    const float dt = steady ? t - h->updated_time : 0.0f;
    k3dom_status s = set_frame_params(h, dt, n);
    if (s != K3DOM_OK) return s;
    if ((s = upload_points(h, xs, ys, zs, n, mem)) != K3DOM_OK) return s;
    cudaError_t e;
    if (steady) {
        if (h->timing || !h->graph_mode) {
            if ((e = enq_frame(h))) return h->fail(e);
        } else {
            if (!h->graph_exec) {
                if ((e = cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal))) return h->fail(e);
                cudaError_t ce = enq_frame(h);
                cudaGraph_t g = nullptr;
                e = cudaStreamEndCapture(h->st, &g);
                if (ce != cudaSuccess) { if (g) cudaGraphDestroy(g); return h->fail(ce); }
                if (e != cudaSuccess) return h->fail(e);
                h->graph = g;
                if ((e = cudaGraphInstantiate(&h->graph_exec, g, 0))) return h->fail(e);
            }
            if ((e = cudaGraphLaunch(h->graph_exec, h->st))) return h->fail(e);
        }
        h->births_done = true;
    } else {
        // DOM::initializeParticles (src/k3dom/dom.cu:52-77; src/dsphdmib/dom.cu:55-82)
        if ((e = enq_occupancy(h, true))) return h->fail(e);
        if ((e = enq_init_particles(h))) return h->fail(e);
    }
    h->shift_pending = false;
    h->pending_shift[0] = h->pending_shift[1] = h->pending_shift[2] = 0;
    h->updated_time = t;
    h->frame += 1;
    if (h->variant == K3DOM_VARIANT_DSPHDMIB) h->iteration += 1;  // src/dsphdmib/dom.cu:52
    h->initialized = true;
    if (!sync) return K3DOM_OK;
    s = finish_sync(h);
    if (s == K3DOM_OK && steady) read_times(h);
    return s;
}

k3dom_status k3dom_update_grid(k3dom_handle* h, float t, const float* xs, const float* ys, const float* zs, int32_t n,
                               k3dom_mem mem) {
    return update_grid_impl(h, t, xs, ys, zs, n, mem, true);
}

k3dom_status k3dom_update_grid_async(k3dom_handle* h, float t, const float* xs, const float* ys, const float* zs,
                                     int32_t n, k3dom_mem mem) {
    return update_grid_impl(h, t, xs, ys, zs, n, mem, false);
}

k3dom_status k3dom_synchronize(k3dom_handle* h) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    k3dom_status s = finish_sync(h);
    if (s == K3DOM_OK) read_times(h);
    return s;
}

k3dom_status k3dom_get_stream(k3dom_handle* h, void** stream) {
    if (!h || !stream) return K3DOM_ERR_INVALID_ARGUMENT;
    *stream = (void*)h->st;
    return K3DOM_OK;
}

k3dom_status k3dom_set_graph_mode(k3dom_handle* h, int enabled) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    h->graph_mode = enabled != 0;
    return K3DOM_OK;
}

k3dom_status k3dom_set_timing(k3dom_handle* h, int enabled) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    h->timing = enabled != 0;
    return K3DOM_OK;
}

k3dom_status k3dom_get_stage_times(k3dom_handle* h, k3dom_stage_times* out) {
    if (!h || !out) return K3DOM_ERR_INVALID_ARGUMENT;
    *out = h->times;
    return K3DOM_OK;
}

// ---- stage calls
#define STAGE_BEGIN                          \
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT; \
    cudaSetDevice(h->device);                \
    cudaError_t e;

k3dom_status k3dom_particle_prediction(k3dom_handle* h, float dt) {
    STAGE_BEGIN
    k3dom_status s = set_frame_params(h, dt, 0);
    if (s != K3DOM_OK) return s;
    if ((e = enq_predict(h))) return h->fail(e);
    h->shift_pending = false;
    h->pending_shift[0] = h->pending_shift[1] = h->pending_shift[2] = 0;
    return finish_sync(h);
}

k3dom_status k3dom_particle_assignment(k3dom_handle* h) {
    STAGE_BEGIN
    if ((e = enq_assign(h))) return h->fail(e);
    return finish_sync(h);
}

k3dom_status k3dom_grid_cell_occupancy_update(k3dom_handle* h, float dt, const float* xs, const float* ys,
                                              const float* zs, int32_t n, k3dom_mem mem) {
    STAGE_BEGIN
    if (n < 0 || (n > 0 && !xs)) return K3DOM_ERR_INVALID_ARGUMENT;
    if (mem == K3DOM_MEM_HOST && n > 0 && has_nonfinite_host(xs, ys, zs, n)) return K3DOM_ERR_INVALID_INPUT;
    k3dom_status s = set_frame_params(h, dt, n);
    if (s != K3DOM_OK) return s;
    if ((s = upload_points(h, xs, ys, zs, n, mem)) != K3DOM_OK) return s;
    if ((e = enq_occupancy(h, false))) return h->fail(e);
    return finish_sync(h);
}

k3dom_status k3dom_update_persistent_particles(k3dom_handle* h) {
    STAGE_BEGIN
    if ((e = enq_persistent(h))) return h->fail(e);
    return finish_sync(h);
}

k3dom_status k3dom_initialize_new_particles(k3dom_handle* h) {
    STAGE_BEGIN
    k3dom_status s = set_frame_params(h, h->fp_host->dt, h->fp_host->n_points);
    if (s != K3DOM_OK) return s;
    if ((e = enq_births(h))) return h->fail(e);
    h->births_done = true;
    return finish_sync(h);
}

k3dom_status k3dom_statistical_moments(k3dom_handle* h) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    return K3DOM_OK;
}

k3dom_status k3dom_resampling(k3dom_handle* h) {
    STAGE_BEGIN
    k3dom_status s = set_frame_params(h, h->fp_host->dt, h->fp_host->n_points);
    if (s != K3DOM_OK) return s;
    if ((e = enq_resample(h, false))) return h->fail(e);
    return finish_sync(h);
}

k3dom_status k3dom_initialize_particles(k3dom_handle* h, const float* xs, const float* ys, const float* zs, int32_t n,
                                        k3dom_mem mem) {
    STAGE_BEGIN
    if (n < 0 || (n > 0 && !xs)) return K3DOM_ERR_INVALID_ARGUMENT;
    if (mem == K3DOM_MEM_HOST && n > 0 && has_nonfinite_host(xs, ys, zs, n)) return K3DOM_ERR_INVALID_INPUT;
    k3dom_status s = set_frame_params(h, 0.0f, n);
    if (s != K3DOM_OK) return s;
    if ((s = upload_points(h, xs, ys, zs, n, mem)) != K3DOM_OK) return s;
    if ((e = enq_occupancy(h, true))) return h->fail(e);
    if ((e = enq_init_particles(h))) return h->fail(e);
    return finish_sync(h);
}

k3dom_status k3dom_finish_frame(k3dom_handle* h, float t) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    h->updated_time = t;
    h->frame += 1;
    if (h->variant == K3DOM_VARIANT_DSPHDMIB) h->iteration += 1;
    h->initialized = true;
    return K3DOM_OK;
}

k3dom_status k3dom_set_frame_index(k3dom_handle* h, int32_t frame) {
    if (!h || frame < 0) return K3DOM_ERR_INVALID_ARGUMENT;
    h->frame = (uint32_t)frame;
    return K3DOM_OK;
}

// ---- info
k3dom_status k3dom_get_info(k3dom_handle* h, k3dom_info* o) {
    if (!h || !o) return K3DOM_ERR_INVALID_ARGUMENT;
    o->grid_size = h->dp.G;
    o->grid_size_z = h->dp.Gz;
    o->grid_cell_count = h->dp.C;
    o->particle_count = h->dp.P;
    o->new_born_particle_count = h->dp.B;
    o->iteration = h->iteration;
    o->variant = (int)h->variant;
    o->initialized = h->initialized ? 1 : 0;
    o->resolution = h->params.resolution;
    o->center_x = h->center_pos[0];
    o->center_y = h->center_pos[1];
    o->center_z = h->center_pos[2];
    o->sensor_x = h->sensor_pos[0];
    o->sensor_y = h->sensor_pos[1];
    o->sensor_z = h->sensor_pos[2];
    o->updated_time = h->updated_time;
    o->max_points = h->rb.max_points;
    o->frame_index = (int32_t)h->frame;
    return K3DOM_OK;
}

k3dom_status k3dom_index_to_coord(k3dom_handle* h, int32_t i, float* x, float* y, float* z) {
    // DOM_c::indexToCoordX/Y/Z (include/common/dom.h:70-81)
    if (!h || i < 0 || i >= h->dp.C) return K3DOM_ERR_INVALID_ARGUMENT;
    const int G = h->dp.G;
    const float r = h->params.resolution;
    if (x) *x = (i % G + 0.5f) * r - h->params.size / 2.0f + h->center_pos[0];
    if (y) *y = ((i % (G * G)) / G + 0.5f) * r - h->params.size / 2.0f + h->center_pos[1];
    if (z) *z = (i / (G * G) + 0.5f) * r - h->params.size_z / 2.0f + h->center_pos[2];
    return K3DOM_OK;
}

// ---- readback
static k3dom_status ensure_export(k3dom_handle* h, size_t bytes) {
    if (h->export_bytes >= bytes) return K3DOM_OK;
    if (h->export_buf) cudaFree(h->export_buf);
    h->export_buf = nullptr;
    h->export_bytes = 0;
    cudaError_t e = cudaMalloc(&h->export_buf, bytes);
    if (e != cudaSuccess) return h->fail(e);
    h->export_bytes = bytes;
    return K3DOM_OK;
}

static k3dom_status deliver(k3dom_handle* h, void* dst, const void* dev_src, size_t bytes, k3dom_mem mem) {
    cudaError_t e = cudaMemcpyAsync(dst, dev_src, bytes,
                                    mem == K3DOM_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, h->st);
    if (e != cudaSuccess) return h->fail(e);
    e = cudaStreamSynchronize(h->st);
    return e == cudaSuccess ? K3DOM_OK : h->fail(e);
}

k3dom_status k3dom_get_cell_field(k3dom_handle* h, k3dom_cell_field field, float* dst, k3dom_mem mem) {
    if (!h || !dst || (int)field < 0 || field >= K3DOM_CELL_FIELD_COUNT) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    const size_t bytes = sizeof(float) * (size_t)h->dp.C;
    float* out = dst;
    if (mem == K3DOM_MEM_HOST) {
        k3dom_status s = ensure_export(h, bytes);
        if (s != K3DOM_OK) return s;
        out = (float*)h->export_buf;
    }
    launch_export_field(h->dp, (int)field, h->cells(), h->cw, h->births_done ? h->born_cum : nullptr, out, h->st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return h->fail(e);
    if (mem == K3DOM_MEM_HOST) return deliver(h, dst, out, bytes, mem);
    e = cudaStreamSynchronize(h->st);
    return e == cudaSuccess ? K3DOM_OK : h->fail(e);
}

k3dom_status k3dom_get_cell_ranges(k3dom_handle* h, int32_t* start, int32_t* end, k3dom_mem mem) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    const size_t bytes = sizeof(int) * (size_t)h->dp.C;
    k3dom_status s = K3DOM_OK;
    if (start) s = deliver(h, start, h->cw.start, bytes, mem);
    if (s == K3DOM_OK && end) s = deliver(h, end, h->cw.end, bytes, mem);
    return s;
}

k3dom_status k3dom_get_gridcell_aos(k3dom_handle* h, void* dst, k3dom_mem mem) {
    if (!h || !dst) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    const size_t bytes = (size_t)K3DOM_GRIDCELL_BYTES * h->dp.C;
    void* out = dst;
    if (mem == K3DOM_MEM_HOST) {
        k3dom_status s = ensure_export(h, bytes);
        if (s != K3DOM_OK) return s;
        out = h->export_buf;
    }
    launch_export_gridcell(h->dp, h->cells(), h->cw, h->births_done ? h->born_cum : nullptr, out, h->st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return h->fail(e);
    if (mem == K3DOM_MEM_HOST) return deliver(h, dst, out, bytes, mem);
    e = cudaStreamSynchronize(h->st);
    return e == cudaSuccess ? K3DOM_OK : h->fail(e);
}

k3dom_status k3dom_get_mappoints(k3dom_handle* h, float* dst, k3dom_mem mem) {
    if (!h || !dst) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    const size_t bytes = sizeof(float) * K3DOM_MAPPOINT_FLOATS * (size_t)h->dp.C;
    float* out = dst;
    if (mem == K3DOM_MEM_HOST) {
        k3dom_status s = ensure_export(h, bytes);
        if (s != K3DOM_OK) return s;
        out = (float*)h->export_buf;
    }
    launch_export_mappoints(h->dp, h->center_pos[0], h->center_pos[1], h->center_pos[2], h->cells(), h->cw, out, h->st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return h->fail(e);
    if (mem == K3DOM_MEM_HOST) return deliver(h, dst, out, bytes, mem);
    e = cudaStreamSynchronize(h->st);
    return e == cudaSuccess ? K3DOM_OK : h->fail(e);
}

k3dom_status k3dom_set_cell_masses(k3dom_handle* h, const float* f, const float* s, const float* d, const float* o,
                                   k3dom_mem mem) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    const size_t bytes = sizeof(float) * (size_t)h->dp.C;
    const cudaMemcpyKind k = mem == K3DOM_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    CellState c = h->cells();
    cudaError_t e;
    if (f && (e = cudaMemcpyAsync(c.free_m, f, bytes, k, h->st))) return h->fail(e);
    if (s && (e = cudaMemcpyAsync(c.static_m, s, bytes, k, h->st))) return h->fail(e);
    if (d && (e = cudaMemcpyAsync(c.dyn_m, d, bytes, k, h->st))) return h->fail(e);
    if (o && (e = cudaMemcpyAsync(c.occ_m, o, bytes, k, h->st))) return h->fail(e);
    e = cudaStreamSynchronize(h->st);
    return e == cudaSuccess ? K3DOM_OK : h->fail(e);
}

static Particles* pick_set(k3dom_handle* h, k3dom_particle_set set, int* n) {
    switch (set) {
        case K3DOM_PARTICLES_PERSISTENT: *n = h->dp.P; return &h->A;
        case K3DOM_PARTICLES_SORTED: *n = h->dp.P; return &h->S;
        case K3DOM_PARTICLES_BIRTH: *n = h->dp.B; return &h->Bp;
    }
    return nullptr;
}

// strips the penalty flag (sign bit) kept in the sorted and birth weights between stages
__global__ void k_abs_copy(const float* __restrict__ src, float* __restrict__ dst, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = fabsf(src[i]);
}

k3dom_status k3dom_get_particles(k3dom_handle* h, k3dom_particle_set set, float* pos, float* vel, float* weight,
                                 int32_t* cell_idx, uint8_t* associated, k3dom_mem mem) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    int n = 0;
    Particles* q = pick_set(h, set, &n);
    if (!q) return K3DOM_ERR_INVALID_ARGUMENT;
    const cudaMemcpyKind k = mem == K3DOM_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    cudaError_t e;
    auto strided = [&](float* dst, const float* a, const float* b, const float* c) -> cudaError_t {
        cudaError_t r;
        if ((r = cudaMemcpy2DAsync(dst, 3 * sizeof(float), a, sizeof(float), sizeof(float), n, k, h->st))) return r;
        if ((r = cudaMemcpy2DAsync(dst + 1, 3 * sizeof(float), b, sizeof(float), sizeof(float), n, k, h->st))) return r;
        return cudaMemcpy2DAsync(dst + 2, 3 * sizeof(float), c, sizeof(float), sizeof(float), n, k, h->st);
    };
    if (pos && (e = strided(pos, q->px, q->py, q->pz))) return h->fail(e);
    if (vel && (e = strided(vel, q->vx, q->vy, q->vz))) return h->fail(e);
    if (weight) {
        k3dom_status s = ensure_export(h, sizeof(float) * (size_t)n);
        if (s != K3DOM_OK) return s;
        ++g_launches;
        k_abs_copy<<<div_up(n, 256), 256, 0, h->st>>>(q->w, (float*)h->export_buf, n);
        if ((e = cudaMemcpyAsync(weight, h->export_buf, sizeof(float) * (size_t)n, k, h->st))) return h->fail(e);
    }
    if (cell_idx && (e = cudaMemcpyAsync(cell_idx, q->cell, sizeof(int) * (size_t)n, k, h->st))) return h->fail(e);
    if (associated && (e = cudaMemcpyAsync(associated, q->assoc, (size_t)n, k, h->st))) return h->fail(e);
    e = cudaStreamSynchronize(h->st);
    return e == cudaSuccess ? K3DOM_OK : h->fail(e);
}

__global__ void k_iota(uint32_t* a, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = (uint32_t)i;
}

k3dom_status k3dom_set_particles(k3dom_handle* h, k3dom_particle_set set, const float* pos, const float* vel,
                                 const float* weight, const int32_t* cell_idx, const uint8_t* associated,
                                 k3dom_mem mem) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    int n = 0;
    Particles* q = pick_set(h, set, &n);
    if (!q) return K3DOM_ERR_INVALID_ARGUMENT;
    if (set == K3DOM_PARTICLES_SORTED && !cell_idx) return K3DOM_ERR_INVALID_ARGUMENT;
    const cudaMemcpyKind k = mem == K3DOM_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    cudaError_t e;
    auto strided = [&](const float* src, float* a, float* b, float* c) -> cudaError_t {
        cudaError_t r;
        if ((r = cudaMemcpy2DAsync(a, sizeof(float), src, 3 * sizeof(float), sizeof(float), n, k, h->st))) return r;
        if ((r = cudaMemcpy2DAsync(b, sizeof(float), src + 1, 3 * sizeof(float), sizeof(float), n, k, h->st))) return r;
        return cudaMemcpy2DAsync(c, sizeof(float), src + 2, 3 * sizeof(float), sizeof(float), n, k, h->st);
    };
    if (pos && (e = strided(pos, q->px, q->py, q->pz))) return h->fail(e);
    if (vel && (e = strided(vel, q->vx, q->vy, q->vz))) return h->fail(e);
    if (weight && (e = cudaMemcpyAsync(q->w, weight, sizeof(float) * (size_t)n, k, h->st))) return h->fail(e);
    if (cell_idx && (e = cudaMemcpyAsync(q->cell, cell_idx, sizeof(int) * (size_t)n, k, h->st))) return h->fail(e);
    if (associated && (e = cudaMemcpyAsync(q->assoc, associated, (size_t)n, k, h->st))) return h->fail(e);
    if (set == K3DOM_PARTICLES_SORTED) {
        // a sorted set defines the cell ranges and sums: rebuild them from it in place
        if ((e = cudaMemcpyAsync(h->sorted_keys, q->cell, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, h->st)))
            return h->fail(e);
        ++g_launches;
        k_iota<<<div_up(n, 256), 256, 0, h->st>>>(h->perm, n);
        if ((e = cudaMemsetAsync(h->cw.start, 0xFF, sizeof(int) * (size_t)h->dp.C, h->st))) return h->fail(e);
        if ((e = cudaMemsetAsync(h->cw.end, 0xFF, sizeof(int) * (size_t)h->dp.C, h->st))) return h->fail(e);
        launch_gather_segsum(h->dp, h->S, h->S, h->sorted_keys, h->perm, h->cw, h->st);
    }
    e = cudaStreamSynchronize(h->st);
    return e == cudaSuccess ? K3DOM_OK : h->fail(e);
}

k3dom_status k3dom_get_sort_permutation(k3dom_handle* h, int32_t* perm, k3dom_mem mem) {
    if (!h || !perm) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    return deliver(h, perm, h->perm, sizeof(int) * (size_t)h->dp.P, mem);
}

k3dom_status k3dom_get_ancestors(k3dom_handle* h, int32_t* anc, k3dom_mem mem) {
    if (!h || !anc) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    return deliver(h, anc, h->ancestors, sizeof(int) * (size_t)h->dp.P, mem);
}

k3dom_status k3dom_get_resampling_state(k3dom_handle* h, float* joint_cum, float* born_cum, float* joint_max,
                                        k3dom_mem mem) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    k3dom_status s = K3DOM_OK;
    if (joint_cum) s = deliver(h, joint_cum, h->joint_cum, sizeof(float) * ((size_t)h->dp.P + h->dp.B), mem);
    if (s == K3DOM_OK && born_cum) s = deliver(h, born_cum, h->born_cum, sizeof(float) * (size_t)h->dp.C, mem);
    if (s == K3DOM_OK && joint_max) s = deliver(h, joint_max, h->joint_max, sizeof(float), mem);
    return s;
}

k3dom_status k3dom_debug_draws(uint64_t seed, int32_t frame, int32_t stage, int64_t first, int64_t count, float* dst,
                               k3dom_mem mem) {
    if (!dst || count < 0 || first < 0 || stage < 1 || stage > 4) return K3DOM_ERR_INVALID_ARGUMENT;
    const int per = stage == 1 ? 6 : (stage == 4 ? 1 : 3);
    const size_t bytes = sizeof(float) * (size_t)count * per;
    float* out = dst;
    cudaError_t e;
    if (mem == K3DOM_MEM_HOST) {
        if ((e = cudaMalloc((void**)&out, std::max<size_t>(bytes, 4)))) return e == cudaErrorMemoryAllocation ? K3DOM_ERR_OUT_OF_MEMORY : K3DOM_ERR_CUDA;
    }
    launch_debug_draws(seed, frame, stage, first, count, out, 0);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess && mem == K3DOM_MEM_HOST) e = cudaMemcpy(dst, out, bytes, cudaMemcpyDeviceToHost);
    if (mem == K3DOM_MEM_HOST) cudaFree(out);
    return e == cudaSuccess ? K3DOM_OK : K3DOM_ERR_CUDA;
}

k3dom_status k3dom_get_diagnostics(k3dom_handle* h, k3dom_diagnostics* out) {
    if (!h || !out) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    DevStatus st;
    cudaError_t e = cudaStreamSynchronize(h->st);
    if (e == cudaSuccess) e = cudaMemcpy(&st, h->status, sizeof(st), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return h->fail(e);
    out->nonfinite_points = (int64_t)st.nonfinite_points;
    out->ray_list_entries = (int64_t)st.ray_entries;
    out->ray_list_capacity = h->rb.capacity;
    out->work_items = (int64_t)st.work_items;
    out->overflow = (int32_t)st.overflow;
    out->kernel_launches_per_frame = h->launches_per_frame;
    out->kernel_evaluations = (int64_t)st.kernel_evals;
    return K3DOM_OK;
}

}  // extern "C"
