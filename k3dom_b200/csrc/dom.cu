// dom.cu -- host orchestration behind the C ABI: the B200 counterpart of dom::DOM_c and the
// two dom::DOM variants (src/common/dom.cu, src/k3dom/dom.cu, src/dsphdmib/dom.cu).
//
// A handle holds S >= 1 independent scenes (a plain handle is a batch of one). Every scene
// owns contiguous ranges of one set of concatenated arrays (cells, particles, births, points,
// evidence tiles), and every stage is ONE launch over all scenes, so a batched frame costs the
// same number of launches as a single one and fills the GPU with the union of the scenes' work.
// Each scene keeps its own parameters, pose, clock and Philox stream (keyed by its own particle
// indices), so a scene updated in a batch gives the same bits as the same scene updated alone.
//
// Differences in structure from the reference, by design:
//  * every buffer is allocated once at creation (the reference allocates measurement arrays,
//    Thrust temporaries and a map copy on every frame);
//  * no host synchronisation inside a frame (the reference reads scalars back at
//    init_new_particles.cu:49, src/common/dom.cu:275 and resampling.cu:58), so the
//    steady-state frame is captured in a CUDA graph and replayed;
//  * particles are double-buffered by role (current / sorted / birth) instead of the deep
//    copy particle_array = particle_array_next (src/k3dom/dom.cu:43);
//  * resampling draws are generated and sorted on a second stream while the evidence
//    kernel runs;
//  * evidence tile shapes and work-item sizes are picked by measuring candidates on live
//    frames (the results do not depend on them).
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

namespace {

// Evidence tiling rules the autotuner chooses from.
enum TileRule { kRuleBySize = 0, kRuleSmall = 1, kRuleFlat = 2, kRuleLarge = 3, kRuleCount = 4 };

TileShape tile_shape(const DevParams& p, int rule) {
    int tx = 8, ty = 8, tz = 4;
    const bool large = (long)p.C >= (1L << 20) && p.Gz >= 8;
    switch (rule) {
        case kRuleBySize: if (large) { tx = 16; ty = 16; tz = 8; } break;
        case kRuleSmall: break;
        case kRuleFlat: tx = 16; ty = 16; tz = 4; break;
        case kRuleLarge: tx = 16; ty = 16; tz = p.Gz >= 8 ? 8 : 4; break;
        default: break;
    }
    TileShape t;
    t.tx = tx; t.ty = ty; t.tz = tz;
    t.ntx = (p.G + tx - 1) / tx;
    t.nty = (p.G + ty - 1) / ty;
    t.ntz = (p.Gz + tz - 1) / tz;
    t.nsbx = tx / 4;
    t.nsby = ty / 4;
    return t;
}

struct SceneHost {
    k3dom_params params{};
    DevParams dp{};
    TileShape ts{};
    float bin_R = 0.0f;
    int max_points = 0;
    // DOM_c host state (include/common/dom.h:135-147)
    bool first_pose_received = false;
    float sensor_pos[3] = {0, 0, 0}, center_pos[3] = {0, 0, 0};
    float updated_time = -1.0f;
    int iteration = 0;
    uint32_t frame = 0;
    bool shift_pending = false;
    int pending_shift[3] = {0, 0, 0};
    bool initialized = false;
    // points arrive in the sensor's own frame: rotate (and translate) them on the device
    bool has_transform = false;
    float rot[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    float trans[3] = {0, 0, 0};
};

int key_bits_for(long n) {
    int b = 1;
    while (b < 31 && (1L << b) < n) ++b;
    return b;
}

}  // namespace

struct k3dom_handle {
    int device = 0;
    int num_sms = 148;
    k3dom_variant variant = K3DOM_VARIANT_K3DOM;
    int S = 1;
    int cur = 0;  // scene the per-scene getters and setters address
    std::vector<SceneHost> sc;
    SceneOffsets off{};
    int P = 0, B = 0, C = 0, N = 0, T = 0;

    cudaStream_t st = nullptr, st2 = nullptr, st3 = nullptr;  // frame; resampling draws; ray lists
    cudaStream_t st4 = nullptr;                               // registered output export
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_bin = nullptr, ev_cells = nullptr;
    cudaEvent_t ev_out = nullptr, ev_out_done = nullptr;
    // registered output (k3dom_set_output): one cell field of one scene, written every frame
    int out_field = -1, out_scene = 0;
    void* out_dst = nullptr;
    k3dom_mem out_mem = K3DOM_MEM_HOST;
    float* out_buf = nullptr;          // device staging when the destination is host memory
    DevStatus* status_host = nullptr;  // pinned copy of the status, read after each frame
    cudaEvent_t ev_t[8] = {};
    bool timing = false;
    k3dom_stage_times times{};

    SceneDev* sc_dev = nullptr;
    SceneOffsets* off_dev = nullptr;
    FrameParams* fp_dev = nullptr;
    FrameParams* fp_host = nullptr;  // pinned, S entries
    DevStatus* status = nullptr;

    Particles A{}, Ss{}, Bp{};
    uint32_t *sorted_keys = nullptr, *perm = nullptr, *alt_k = nullptr, *alt_v = nullptr;
    // The persistent set lives in A (structure of arrays; written by resampling, the first frame
    // and k3dom_set_particles) and, after prediction, in 32-byte records X (what the assignment
    // gathers). Which of the two holds the current set is tracked at enqueue time; every full
    // frame ends with A current, so a captured frame's replays leave both flags as they were.
    float4* X = nullptr;
    bool a_current = true;   // A holds the current persistent set
    bool x_current = false;  // X holds it
    SegRec* seg_rec = nullptr;  // piece sums of the segmented per-cell sums, one per 128 sorted slots
    int2* res_br = nullptr;     // ancestor brackets of the resampling blocks
    uint32_t* os_scratch = nullptr;  // onesweep particle sort: histograms and tile status
    long os_words = 0;
    SortWait sort_wait;
    CellState cs[2]{};  // cs[0] live, cs[1] spare for the map shift
    int *start2 = nullptr, *end2 = nullptr;
    CellWork cw{};
    float *born_cum = nullptr, *joint_cum = nullptr, *joint_max = nullptr;
    void* exact_scratch = nullptr;
    ExactTile *plan_born = nullptr, *plan_joint = nullptr;
    int plan_born_n = 0, plan_joint_n = 0;
    uint32_t *draw_keys = nullptr, *draw_sorted = nullptr, *draw_alt = nullptr;
    uint32_t* os_draw = nullptr;  // onesweep scratch of the draw sort (runs on the second stream)
    long os_draw_words = 0;
    cudaEvent_t ev_staged = nullptr;  // host staging (frame scalars, points) consumed
    int* ancestors = nullptr;
    float* pts = nullptr;  // device x | y | z, N slots each
    float* pts_pinned = nullptr;
    float* pts_xyz = nullptr;         // device staging of interleaved scans (3 N floats)
    float* pts_xyz_pinned = nullptr;  // pinned host staging of interleaved scans (3 N floats)
    RayBuffers rb{};
    std::vector<void*> ray_allocs;  // buffers sized by points and tiles (re-made on growth)
    void* export_buf = nullptr;
    size_t export_bytes = 0;
    std::vector<void*> allocs;

    bool births_done = false;
    int launches_per_frame = 0;
    int launches_upload = 0;  // kernels of the last frame's point upload (de-interleaving)
    int ds_sized_chunk = 0;  // chunk the DS count buffer was sized for

    // evidence tuning
    int tile_rule = kRuleBySize;
    int chunk = 1024;
    int tune_next = -1;  // next candidate to measure, -1 when not tuning
    float tune_best_ms = 0.0f;
    int tune_best = 0, tuned = 0;
    std::vector<float> tune_ms;

    // graph of the steady-state frame
    bool graph_mode = true;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;

    cudaError_t last_error = cudaSuccess;
    k3dom_status fail(cudaError_t e) {
        last_error = e;
        return e == cudaErrorMemoryAllocation ? K3DOM_ERR_OUT_OF_MEMORY : K3DOM_ERR_CUDA;
    }

    template <typename T>
    cudaError_t alloc(T** p, size_t count, bool zero = true, std::vector<void*>* list = nullptr) {
        *p = nullptr;
        if (count == 0) count = 1;
        cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
        if (e != cudaSuccess) return e;
        (list ? list : &allocs)->push_back((void*)*p);
        // zero on the handle's stream: it is non-blocking, so a memset on the legacy default stream
        // would not be ordered before the handle's own work on the buffer
        if (zero) e = cudaMemsetAsync(*p, 0, count * sizeof(T), st);
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
    void drop_graph() {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        if (graph) cudaGraphDestroy(graph);
        graph_exec = nullptr;
        graph = nullptr;
    }
    void free_ray_buffers() {
        if (rb.ktex) cudaDestroyTextureObject(rb.ktex);
        rb.ktex = 0;
        for (void* p : ray_allocs) cudaFree(p);
        ray_allocs.clear();
        if (pts_pinned) cudaFreeHost(pts_pinned);
        pts_pinned = nullptr;
        if (pts_xyz_pinned) cudaFreeHost(pts_xyz_pinned);
        pts_xyz_pinned = nullptr;
    }
    void release() {
        drop_graph();
        free_ray_buffers();
        for (void* p : allocs) cudaFree(p);
        allocs.clear();
        if (fp_host) cudaFreeHost(fp_host);
        if (status_host) cudaFreeHost(status_host);
        if (export_buf) cudaFree(export_buf);
        if (out_buf) cudaFree(out_buf);
        for (auto& e : ev_t)
            if (e) cudaEventDestroy(e);
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (ev_bin) cudaEventDestroy(ev_bin);
        if (ev_cells) cudaEventDestroy(ev_cells);
        if (ev_staged) cudaEventDestroy(ev_staged);
        if (ev_out) cudaEventDestroy(ev_out);
        if (ev_out_done) cudaEventDestroy(ev_out_done);
        if (st) cudaStreamDestroy(st);
        if (st2) cudaStreamDestroy(st2);
        if (st3) cudaStreamDestroy(st3);
        if (st4) cudaStreamDestroy(st4);
    }
    CellState cells() const { return cs[0]; }
    Batch batch() const {
        Batch b;
        b.S = S;
        b.variant = (int)variant;
        b.P = P; b.B = B; b.C = C; b.N = N; b.T = T;
        b.sc = sc_dev;
        b.fp = fp_dev;
        b.off = off_dev;
        return b;
    }
    bool ds() const { return variant == K3DOM_VARIANT_DSPHDMIB; }
};

namespace {

CellState offset_cells(CellState c, long o) {
    c.free_m += o; c.static_m += o; c.dyn_m += o; c.occ_m += o; c.pers_m += o; c.pred_m += o; c.born_m += o;
    c.mvx += o; c.mvy += o; c.mvz += o;
    return c;
}
CellWork offset_work(CellWork w, long o) {
    w.start += o; w.end += o; w.sum_w += o; w.sum_wvx += o; w.sum_wvy += o; w.sum_wvz += o; w.factor += o;
    w.divisor += o; w.meas_occ += o; w.meas_free += o; w.del_occ += o; w.del_free += o;
    return w;
}
Particles offset_particles(Particles q, long o) {
    q.px += o; q.py += o; q.pz += o; q.vx += o; q.vy += o; q.vz += o; q.w += o; q.cell += o; q.assoc += o;
    return q;
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

DevParams dev_params(const k3dom_params& p, k3dom_variant variant) {
    DevParams d{};
    d.G = static_cast<int>(p.size / p.resolution);  // src/common/dom.cu:30
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
    return d;
}

// Point slots and evidence tiles of every scene; uploads the scene table and kernel tables.
cudaError_t layout_points_tiles(k3dom_handle* h) {
    int pt = 0, tl = 0;
    for (int s = 0; s < h->S; ++s) {
        SceneHost& x = h->sc[s];
        x.ts = tile_shape(x.dp, h->tile_rule);
        h->off.point[s] = pt;
        h->off.tile[s] = tl;
        pt += x.max_points;
        tl += x.ts.ntx * x.ts.nty * x.ts.ntz;
    }
    h->off.point[h->S] = pt;
    h->off.tile[h->S] = tl;
    h->N = pt;
    h->T = tl;
    std::vector<SceneDev> sd(h->S);
    std::vector<float4> tabs((size_t)h->S * kKernelTableSize);
    for (int s = 0; s < h->S; ++s) {
        SceneHost& x = h->sc[s];
        SceneDev& d = sd[s];
        std::memset(&d, 0, sizeof(d));
        d.p = x.dp;
        d.ts = x.ts;
        d.cell_off = h->off.cell[s];
        d.part_off = h->off.part[s];
        d.birth_off = h->off.birth[s];
        d.joint_off = h->off.joint[s];
        d.point_off = h->off.point[s];
        d.tile_off = h->off.tile[s];
        d.n_tiles = h->off.tile[s + 1] - h->off.tile[s];
        d.max_points = x.max_points;
        fill_scene_evidence(d, h->ds(), tabs.data() + (size_t)s * kKernelTableSize);
        x.bin_R = d.bin_R;
    }
    cudaError_t e;
    // on the handle's stream (ordered before its kernels), then waited for: the sources are locals
    if ((e = cudaMemcpyAsync(h->sc_dev, sd.data(), sizeof(SceneDev) * sd.size(), cudaMemcpyHostToDevice, h->st)))
        return e;
    if ((e = cudaMemcpyAsync(h->off_dev, &h->off, sizeof(SceneOffsets), cudaMemcpyHostToDevice, h->st))) return e;
    if (h->rb.ktab &&
        (e = cudaMemcpyAsync(h->rb.ktab, tabs.data(), sizeof(float4) * tabs.size(), cudaMemcpyHostToDevice, h->st)))
        return e;
    return cudaStreamSynchronize(h->st);
}

static cudaError_t alloc_points(k3dom_handle* h);

// Buffers sized by the point slots and tiles: ray data, entry lists, tile lists, points.
cudaError_t alloc_ray_buffers(k3dom_handle* h) {
    h->drop_graph();
    h->free_ray_buffers();
    RayBuffers& rb = h->rb;
    rb = RayBuffers{};
    std::vector<void*>* L = &h->ray_allocs;
    cudaError_t e;
    if ((e = h->alloc(&rb.ktab, (size_t)h->S * kKernelTableSize, true, L))) return e;
    if ((e = make_kernel_table_texture(rb, h->S))) return e;
    if ((e = layout_points_tiles(h))) return e;
    long cap = 0;
    for (int s = 0; s < h->S; ++s)
        cap += ray_entries_bound(h->sc[s].dp, h->sc[s].ts, h->sc[s].max_points, h->sc[s].bin_R);
    cap = std::max(cap, 4096L);
    if (cap > 0xFFFFFFF0L) cap = 0xFFFFFFF0L;
    rb.capacity = cap;
    rb.chunk = h->chunk;
    const int N = h->N, T = h->T;
    if ((e = h->alloc(&rb.ray_a, N, true, L)) || (e = h->alloc(&rb.ray_c, N, true, L)) ||
        (e = h->alloc(&rb.counts, (size_t)kRayThreads * N, true, L)) || (e = h->alloc(&rb.evals2, cap, false, L)) ||
        (e = h->alloc(&rb.tile_start, T + 1, true, L)) || (e = h->alloc(&rb.item_off, T + 1, true, L)) ||
        (e = h->alloc(&rb.tile_done, T, true, L)) || (e = h->alloc(&rb.acc, 2 * (size_t)h->C, true, L)) ||
        (e = h->alloc(&rb.total, 4, true, L)))
        return e;
    if (placed_lists(h->ds(), T)) {  // per-tile tallies and per-block offsets
        if ((e = h->alloc(&rb.tile_tally, T, true, L)) ||
            (e = h->alloc(&rb.block_base, (size_t)bin_blocks((long)kRayThreads * N) * T, true, L)))
            return e;
        return alloc_points(h);
    }
    // sorted lists: entries in ray order, sorted by tile with their own sort/scan scratch (the
    // lists are built beside the particle sort)
    if ((e = h->alloc(&rb.offsets, N, true, L)) || (e = h->alloc(&rb.ekeys, cap, false, L)) ||
        (e = h->alloc(&rb.evals, cap, false, L)) || (e = h->alloc(&rb.ekeys2, cap, false, L)) ||
        (e = h->alloc(&rb.tile_items, T, true, L)))
        return e;
    int bits = 1;
    while ((1 << bits) < T + 1) ++bits;
    int pb[8];
    if (onesweep_plan(bits, pb) > 1) {
        if ((e = h->alloc(&rb.ekeys_alt, cap, false, L)) || (e = h->alloc(&rb.evals_alt, cap, false, L))) return e;
    } else {
        rb.ekeys_alt = rb.ekeys;
        rb.evals_alt = rb.evals;
    }
    if (h->ds()) {
        h->ds_sized_chunk = std::max(32, h->chunk);
        const long items_max = T + cap / h->ds_sized_chunk + 2;
        rb.ds_count_capacity = ds_count_bytes(items_max);
        if ((e = h->alloc(&rb.ds_counts, rb.ds_count_capacity, true, L))) return e;
    }
    rb.os_words = onesweep_scratch_words(cap, bits);
    rb.scan_words = scan_u32_tiles(std::max((long)N, (long)T + 1)) + 16;
    if ((e = h->alloc(&rb.os_scratch, rb.os_words, true, L))) return e;
    if ((e = h->alloc(&rb.scan_tmp, rb.scan_words, true, L))) return e;
    return alloc_points(h);
}

// The frame's point buffers: device scan (de-interleaved), its (x, y, z) upload and pinned staging.
static cudaError_t alloc_points(k3dom_handle* h) {
    const int N = h->N;
    std::vector<void*>* L = &h->ray_allocs;
    cudaError_t e;
    if ((e = h->alloc(&h->pts, 3 * (size_t)N, true, L))) return e;
    if ((e = h->alloc(&h->pts_xyz, 3 * (size_t)N, true, L))) return e;
    if ((e = cudaMallocHost((void**)&h->pts_pinned, 3 * (size_t)N * sizeof(float)))) return e;
    if ((e = cudaMallocHost((void**)&h->pts_xyz_pinned, 3 * (size_t)N * sizeof(float)))) return e;
    return cudaSuccess;
}

}  // namespace

// ===================================================================== frame pieces
namespace {

// Frame scalars of every scene (dt[s], n[s]); waits until the previous staging was consumed.
k3dom_status set_frame_params(k3dom_handle* h, const float* dt, const int* n_points) {
    cudaError_t e = cudaEventSynchronize(h->ev_staged);
    if (e != cudaSuccess) return h->fail(e);
    for (int s = 0; s < h->S; ++s) {
        const SceneHost& x = h->sc[s];
        FrameParams& f = h->fp_host[s];
        f.dt = dt[s];
        f.gamma_dt = std::pow((double)x.dp.gamma, (double)dt[s]);
        f.sensor_x = x.sensor_pos[0] - x.center_pos[0];
        f.sensor_y = x.sensor_pos[1] - x.center_pos[1];
        f.sensor_z = x.sensor_pos[2] - x.center_pos[2];
        f.n_points = n_points[s];
        f.frame = x.frame;
        f.shift_x = x.pending_shift[0];
        f.shift_y = x.pending_shift[1];
        f.shift_z = x.pending_shift[2];
        f.shift_pending = x.shift_pending ? 1 : 0;
        f.seed = x.params.seed;
        f.has_transform = x.has_transform ? 1 : 0;
        std::memcpy(f.rot, x.rot, sizeof(f.rot));
        std::memcpy(f.trans, x.trans, sizeof(f.trans));
    }
    e = cudaMemcpyAsync(h->fp_dev, h->fp_host, sizeof(FrameParams) * h->S, cudaMemcpyHostToDevice, h->st);
    if (e != cudaSuccess) return h->fail(e);
    e = cudaEventRecord(h->ev_staged, h->st);
    return e == cudaSuccess ? K3DOM_OK : h->fail(e);
}

// Same dt and point count for every scene (the stage calls).
k3dom_status set_frame_params_all(k3dom_handle* h, float dt, int n) {
    std::vector<float> d(h->S, dt);
    std::vector<int> m(h->S, n);
    return set_frame_params(h, d.data(), m.data());
}

// Point capacities grow (allocation happens only here, outside the steady state).
k3dom_status grow_points(k3dom_handle* h, const int32_t* n) {
    bool grow = false;
    for (int s = 0; s < h->S; ++s) grow = grow || n[s] > h->sc[s].max_points;
    if (!grow) return K3DOM_OK;
    cudaError_t e = cudaStreamSynchronize(h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st2);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st3);
    if (e != cudaSuccess) return h->fail(e);
    for (int s = 0; s < h->S; ++s) {
        SceneHost& x = h->sc[s];
        if (n[s] > x.max_points) x.max_points = std::max(n[s], (int)(x.max_points * 1.25));
        x.params.max_points = x.max_points;
    }
    long slots = 0;
    for (int s = 0; s < h->S; ++s) slots += h->sc[s].max_points;
    if (slots > (1L << 30)) return K3DOM_ERR_CAPACITY;
    e = alloc_ray_buffers(h);
    if (e != cudaSuccess) return h->fail(e);
    e = cudaEventRecord(h->ev_staged, h->st);
    return e == cudaSuccess ? K3DOM_OK : h->fail(e);
}

// A float is infinite or NaN exactly when its exponent bits are all ones; the branch-free OR
// over the bits lets the compiler vectorise the scan.
static bool nonfinite_any(const float* v, long m) {
    uint32_t bad = 0;
    for (long i = 0; i < m; ++i) {
        uint32_t u;
        std::memcpy(&u, v + i, sizeof(u));
        bad |= (uint32_t)((u & 0x7F800000u) == 0x7F800000u);
    }
    return bad != 0;
}

// Copy m floats and report whether any of them is non-finite, in one pass over the source.
static bool copy_nonfinite_any(float* __restrict__ dst, const float* __restrict__ v, long m) {
    uint32_t bad = 0;
    for (long i = 0; i < m; ++i) {
        uint32_t u;
        std::memcpy(&u, v + i, sizeof(u));
        std::memcpy(dst + i, &u, sizeof(u));
        bad |= (uint32_t)((u & 0x7F800000u) == 0x7F800000u);
    }
    return bad != 0;
}

bool has_nonfinite_host(const float* xs, const float* ys, const float* zs, int n) {
    const bool inter = (ys == nullptr || zs == nullptr);
    if (inter) return nonfinite_any(xs, 3L * n);
    return nonfinite_any(xs, n) || nonfinite_any(ys, n) || nonfinite_any(zs, n);
}

// (x, y, z) interleaved -> the three point planes
__global__ void k_deinterleave(const float* __restrict__ xyz, int n, float* __restrict__ x, float* __restrict__ y,
                               float* __restrict__ z) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x[i] = xyz[3 * i];
    y[i] = xyz[3 * i + 1];
    z[i] = xyz[3 * i + 2];
}

static cudaError_t deinterleave(k3dom_handle* h, const float* xyz, int n, float* dx, float* dy, float* dz) {
    ++g_launches;
    k_deinterleave<<<div_up(n, 256), 256, 0, h->st>>>(xyz, n, dx, dy, dz);
    return cudaGetLastError();
}

static bool is_pinned_host(const void* p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();  // unregistered pageable memory on older drivers
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Points of scene s -> device SoA slots of the scene, in two phases. kStage starts the upload
// of an interleaved host scan into device staging (straight from the caller's memory when it is
// pinned and the call waits for the frame, so the caller cannot reuse the buffer while the copy
// is pending; otherwise through pinned memory, whose previous use set_frame_params waited on);
// the host's finiteness check runs while that copy is in flight, or during the copy into pinned
// memory, which then sets *checked and *nonfinite. kPlace writes the planes: de-interleaving on
// the device, or copies of separate x/y/z arrays.
enum UploadPhase { kStage, kPlace };

k3dom_status upload_points(k3dom_handle* h, int s, const float* xs, const float* ys, const float* zs, int n,
                           k3dom_mem mem, bool sync, UploadPhase phase, bool* checked = nullptr,
                           bool* nonfinite = nullptr) {
    if (n == 0) return K3DOM_OK;
    const long N = h->N, o = h->off.point[s];
    float* dx = h->pts + o;
    float* dy = h->pts + N + o;
    float* dz = h->pts + 2 * N + o;
    const bool interleaved = (ys == nullptr || zs == nullptr);
    cudaError_t e;
    if (mem == K3DOM_MEM_HOST && interleaved) {
        if (phase == kStage) {
            const float* src = xs;
            if (!sync || !is_pinned_host(xs)) {
                const bool bad = copy_nonfinite_any(h->pts_xyz_pinned + 3 * o, xs, 3L * n);
                if (checked) *checked = true;
                if (nonfinite) *nonfinite = bad;
                src = h->pts_xyz_pinned + 3 * o;
            }
            if ((e = cudaMemcpyAsync(h->pts_xyz + 3 * o, src, 3 * n * sizeof(float), cudaMemcpyHostToDevice,
                                     h->st)) ||
                (e = cudaEventRecord(h->ev_staged, h->st)))
                return h->fail(e);
            return K3DOM_OK;
        }
        if ((e = deinterleave(h, h->pts_xyz + 3 * o, n, dx, dy, dz))) return h->fail(e);
        return K3DOM_OK;
    }
    if (phase == kStage) return K3DOM_OK;
    if (mem == K3DOM_MEM_HOST) {
        float* hx = h->pts_pinned + o;
        float* hy = h->pts_pinned + N + o;
        float* hz = h->pts_pinned + 2 * N + o;
        std::memcpy(hx, xs, n * sizeof(float));
        std::memcpy(hy, ys, n * sizeof(float));
        std::memcpy(hz, zs, n * sizeof(float));
        if ((e = cudaMemcpyAsync(dx, hx, n * sizeof(float), cudaMemcpyHostToDevice, h->st)) ||
            (e = cudaMemcpyAsync(dy, hy, n * sizeof(float), cudaMemcpyHostToDevice, h->st)) ||
            (e = cudaMemcpyAsync(dz, hz, n * sizeof(float), cudaMemcpyHostToDevice, h->st)) ||
            (e = cudaEventRecord(h->ev_staged, h->st)))
            return h->fail(e);
    } else if (interleaved) {
        if ((e = deinterleave(h, xs, n, dx, dy, dz))) return h->fail(e);
    } else {
        if ((e = cudaMemcpyAsync(dx, xs, n * sizeof(float), cudaMemcpyDeviceToDevice, h->st)) ||
            (e = cudaMemcpyAsync(dy, ys, n * sizeof(float), cudaMemcpyDeviceToDevice, h->st)) ||
            (e = cudaMemcpyAsync(dz, zs, n * sizeof(float), cudaMemcpyDeviceToDevice, h->st)))
            return h->fail(e);
    }
    return K3DOM_OK;
}

// Every scene's points: stage, check host scans for non-finite coordinates (refused before
// anything reads the staging), place.
k3dom_status upload_all(k3dom_handle* h, const float* const* xs, const float* const* ys, const float* const* zs,
                        const int32_t* n, k3dom_mem mem, bool sync, bool check) {
    k3dom_status st;
    std::vector<char> checked(h->S, 0);
    for (int s = 0; s < h->S; ++s) {
        bool done = false, bad = false;
        if ((st = upload_points(h, s, xs[s], ys ? ys[s] : nullptr, zs ? zs[s] : nullptr, n[s], mem, sync, kStage,
                                &done, &bad)))
            return st;
        if (check && bad) return K3DOM_ERR_INVALID_INPUT;
        checked[s] = done;
    }
    if (check && mem == K3DOM_MEM_HOST)
        for (int s = 0; s < h->S; ++s)
            if (n[s] > 0 && !checked[s] &&
                has_nonfinite_host(xs[s], ys ? ys[s] : nullptr, zs ? zs[s] : nullptr, n[s]))
                return K3DOM_ERR_INVALID_INPUT;
    for (int s = 0; s < h->S; ++s)
        if ((st = upload_points(h, s, xs[s], ys ? ys[s] : nullptr, zs ? zs[s] : nullptr, n[s], mem, sync, kPlace)))
            return st;
    return K3DOM_OK;
}

// Arguments only; host scans are checked for non-finite coordinates while they upload (upload_all).
k3dom_status check_points(const float* xs, const float* ys, const float* zs, int n, k3dom_mem mem) {
    (void)ys;
    (void)zs;
    (void)mem;
    if (n < 0 || (n > 0 && !xs)) return K3DOM_ERR_INVALID_ARGUMENT;
    return K3DOM_OK;
}

void rec(k3dom_handle* h, int i) {
    if (h->timing) cudaEventRecord(h->ev_t[i], h->st);
}

// --- enqueue helpers (no synchronisation) ---
// The persistent set as structure of arrays in A (unpacked from X when prediction left it there).
cudaError_t ensure_a_current(k3dom_handle* h) {
    if (h->a_current) return cudaSuccess;
    launch_unpack_records(h->P, h->X, h->A, h->st);
    h->a_current = true;
    return cudaGetLastError();
}

cudaError_t enq_predict(k3dom_handle* h) {
    cudaError_t e = ensure_a_current(h);
    if (e != cudaSuccess) return e;
    launch_predict(h->batch(), h->A, h->X, h->st);
    h->a_current = false;
    h->x_current = true;
    return cudaGetLastError();
}

cudaError_t enq_assign(k3dom_handle* h) {
    // the records the gather reads (prediction wrote them; otherwise packed from A, whose cell
    // indices are always current)
    if (!h->x_current) {
        launch_pack_records(h->P, h->A, h->X, h->st);
        h->x_current = true;
    }
    cudaError_t e = onesweep_sort_pairs(reinterpret_cast<const uint32_t*>(h->A.cell), nullptr, h->sorted_keys,
                                        h->perm, h->alt_k, h->alt_v, h->P, key_bits_for(h->C), h->os_scratch,
                                        h->os_words, h->status, h->sort_wait, h->st);
    if (e != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(h->cw.start, 0xFF, sizeof(int) * (size_t)h->C, h->st))) return e;
    if ((e = cudaMemsetAsync(h->cw.end, 0xFF, sizeof(int) * (size_t)h->C, h->st))) return e;
    launch_gather_segsum(h->batch(), h->X, h->Ss, h->sorted_keys, h->perm, h->cw, h->seg_rec, h->st);
    return cudaGetLastError();
}

cudaError_t enq_binning(k3dom_handle* h, cudaStream_t s) {
    const long N = h->N;
    return build_ray_lists(h->batch(), h->pts, h->pts + N, h->pts + 2 * N, h->rb, h->ds(), h->status, h->sort_wait,
                           s);
}

cudaError_t enq_evidence(k3dom_handle* h, bool first_frame) {
    const Batch bt = h->batch();
    if (h->ds())
        return launch_ds_evidence(bt, h->rb, h->cells(), h->cw, first_frame, h->status, h->st);
    return launch_k3dom_evidence(bt, h->rb, h->cells(), h->cw, first_frame, h->status, h->st);
}

cudaError_t enq_occupancy(k3dom_handle* h, bool first_frame) {
    cudaError_t e = enq_binning(h, h->st);
    if (e != cudaSuccess) return e;
    rec(h, 7);
    return enq_evidence(h, first_frame);
}

cudaError_t enq_persistent(k3dom_handle* h, cudaStream_t s) {
    launch_reweight(h->batch(), h->Ss, h->sorted_keys, h->cw, s);
    return cudaGetLastError();
}

cudaError_t enq_births(k3dom_handle* h) {
    cudaError_t e = exact_scan_plan(h->plan_born, h->plan_born_n, h->exact_scratch, h->st);
    if (e != cudaSuccess) return e;
    launch_births(h->batch(), h->cells().born_m, h->born_cum, h->Bp, h->st);
    return cudaGetLastError();
}

cudaError_t enq_draws(k3dom_handle* h, cudaStream_t s) {
    launch_draw_keys(h->batch(), h->draw_keys, s);
    SortWait w = h->sort_wait;
    w.skip_tile = -1;
    return onesweep_sort_pairs(h->draw_keys, nullptr, h->draw_sorted, nullptr, h->draw_alt, nullptr, h->P,
                               draw_key_bits(h->S), h->os_draw, h->os_draw_words, h->status, w, s);
}

cudaError_t enq_resample(k3dom_handle* h, bool draws_ready) {
    cudaError_t e;
    if (!draws_ready) {
        if ((e = enq_draws(h, h->st))) return e;
    }
    // the joint weights' prefix; the penalised (sign-bit) weights count as 0 and are cleared
    if ((e = exact_scan_plan(h->plan_joint, h->plan_joint_n, h->exact_scratch, h->st, true))) return e;
    launch_resample(h->batch(), h->joint_cum, h->draw_sorted, h->Ss, h->Bp, h->A, h->ancestors, h->joint_max,
                    h->res_br, h->st);
    h->a_current = true;
    h->x_current = false;
    return cudaGetLastError();
}

cudaError_t enq_init_particles(k3dom_handle* h) {
    cudaError_t e = exact_scan_plan(h->plan_born, h->plan_born_n, h->exact_scratch, h->st);
    if (e != cudaSuccess) return e;
    launch_init_particles(h->batch(), h->born_cum, h->A, h->st);
    h->a_current = true;
    h->x_current = false;
    return cudaGetLastError();
}

// Registered output: the field of the chosen scene is exported on a side stream as soon as the
// stage it depends on has run (the cell update for masses, velocities, evidence and reweight
// factors; the births' scan for w_A / w_UA), so its copy overlaps the rest of the frame. The frame
// joins it at its end (enq_output_join).
bool output_needs_births(int field) { return field == 12 || field == 13; }

cudaError_t enq_output(k3dom_handle* h) {
    if (h->out_field < 0 || !h->out_dst) return cudaSuccess;
    const int s = h->out_scene;
    const SceneHost& x = h->sc[s];
    const long co = h->off.cell[s];
    cudaError_t e;
    if ((e = cudaEventRecord(h->ev_out, h->st)) || (e = cudaStreamWaitEvent(h->st4, h->ev_out, 0))) return e;
    float* dev = h->out_mem == K3DOM_MEM_HOST ? h->out_buf : static_cast<float*>(h->out_dst);
    launch_export_field(x.dp, h->out_field, offset_cells(h->cells(), co), offset_work(h->cw, co),
                        h->born_cum + co, h->off.part[s], dev, h->st4);
    if ((e = cudaGetLastError())) return e;
    if (h->out_mem == K3DOM_MEM_HOST &&
        (e = cudaMemcpyAsync(h->out_dst, dev, sizeof(float) * (size_t)x.dp.C, cudaMemcpyDeviceToHost, h->st4)))
        return e;
    return cudaEventRecord(h->ev_out_done, h->st4);
}

cudaError_t enq_output_join(k3dom_handle* h) {
    if (h->out_field < 0 || !h->out_dst) return cudaSuccess;
    return cudaStreamWaitEvent(h->st, h->ev_out_done, 0);
}

// The steady-state frame (DOM::updateGrid's branch for updated_time > 0), all scenes.
cudaError_t enq_frame(k3dom_handle* h) {
    cudaError_t e;
    const long l0 = g_launches;
    // resampling draws depend only on (seed, frame): produce them beside the frame
    if ((e = cudaEventRecord(h->ev_fork, h->st))) return e;
    if ((e = cudaStreamWaitEvent(h->st2, h->ev_fork, 0))) return e;
    if ((e = enq_draws(h, h->st2))) return e;
    if ((e = cudaEventRecord(h->ev_join, h->st2))) return e;
    // the ray lists depend on the points only: built beside prediction and assignment, except
    // when each stage is timed on its own. K3DOM's evidence needs only the lists, so it runs there
    // too, and the cells are updated once both sides are done; DS's evidence pass needs the
    // particles' per-cell counts throughout and follows assignment.
    const bool overlap = !h->timing;
    const bool split = overlap && !h->ds();
    if (overlap) {
        if ((e = cudaStreamWaitEvent(h->st3, h->ev_fork, 0))) return e;
        if ((e = enq_binning(h, h->st3))) return e;
        if (split && (e = launch_k3dom_evidence(h->batch(), h->rb, h->cells(), h->cw, false, h->status, h->st3,
                                                false)))
            return e;
        if ((e = cudaEventRecord(h->ev_bin, h->st3))) return e;
    }
    rec(h, 0);
    if ((e = enq_predict(h))) return e;
    rec(h, 1);
    if ((e = enq_assign(h))) return e;
    rec(h, 2);
    if (split) {
        if ((e = cudaStreamWaitEvent(h->st, h->ev_bin, 0))) return e;
        if ((e = launch_k3dom_update_cells(h->batch(), h->rb, h->cells(), h->cw, h->status, h->st))) return e;
    } else if (overlap) {
        if ((e = cudaStreamWaitEvent(h->st, h->ev_bin, 0))) return e;
        if ((e = enq_evidence(h, false))) return e;
    } else if ((e = enq_occupancy(h, false))) {
        return e;
    }
    rec(h, 3);
    if (!output_needs_births(h->out_field) && (e = enq_output(h))) return e;
    if (overlap) {
        // the reweight needs the cells' factors only, the births the born masses: the reweight
        // runs on the draws' stream beside the births, and resampling waits for both
        if ((e = cudaEventRecord(h->ev_cells, h->st)) || (e = cudaStreamWaitEvent(h->st2, h->ev_cells, 0)) ||
            (e = enq_persistent(h, h->st2)) || (e = cudaEventRecord(h->ev_join, h->st2)))
            return e;
    } else if ((e = enq_persistent(h, h->st))) {
        return e;
    }
    rec(h, 4);
    if ((e = enq_births(h))) return e;
    rec(h, 5);
    if (output_needs_births(h->out_field) && (e = enq_output(h))) return e;
    if ((e = cudaStreamWaitEvent(h->st, h->ev_join, 0))) return e;
    if ((e = enq_resample(h, true))) return e;
    if ((e = enq_output_join(h))) return e;
    rec(h, 6);
    h->launches_per_frame = (int)(g_launches - l0);
    return cudaSuccess;
}

void read_times(k3dom_handle* h) {
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

// Evidence tuning: candidates are (tile rule, chunk) pairs measured one per steady frame.
// (256-ray items, the 128-thread evidence build, are left out: on a 256x256x32-voxel scene with
// 120,000-point scans the one-frame measurements put 16x16x4 tiles at 256 rays ahead of 512 while
// the steady graph-replayed frame is 5 % slower with them; set them with k3dom_set_tuning.)
constexpr int kTuneChunks[2] = {512, 1024};
constexpr int kTuneCount = kRuleCount * 2;
static_assert(kTuneCount <= K3DOM_TUNE_MAX_CANDIDATES, "tuning candidates");

cudaError_t apply_tuning(k3dom_handle* h, int rule, int chunk) {
    if (rule == h->tile_rule && chunk == h->chunk) return cudaSuccess;
    cudaError_t e = cudaStreamSynchronize(h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st2);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st3);
    if (e != cudaSuccess) return e;
    // a smaller chunk makes more work items than the DS count buffer was sized for
    const bool relayout = rule != h->tile_rule || (h->ds() && chunk < h->ds_sized_chunk);
    h->tile_rule = rule;
    h->chunk = chunk;
    h->drop_graph();
    if (relayout) {
        e = alloc_ray_buffers(h);
        if (e == cudaSuccess) e = cudaEventRecord(h->ev_staged, h->st);
        return e;
    }
    h->rb.chunk = chunk;
    return cudaSuccess;
}

}  // namespace

// ===================================================================== C ABI
extern "C" {

static cudaError_t copy_cells_back(k3dom_handle* h, int s);

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

const char* k3dom_last_cuda_error(k3dom_handle* h) {
    if (!h) return "no handle";
    return cudaGetErrorString(h->last_error);
}

k3dom_status k3dom_batch_create(const k3dom_params* params, int32_t n_scenes, k3dom_variant variant, int device,
                                k3dom_handle** out) {
    if (!out) return K3DOM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (!params || n_scenes < 1) return K3DOM_ERR_INVALID_ARGUMENT;
    if (n_scenes > kMaxScenes) return K3DOM_ERR_CAPACITY;
    long tp = 0, tb = 0, tc = 0;
    for (int s = 0; s < n_scenes; ++s) {
        k3dom_status v = validate(&params[s], variant);
        if (v != K3DOM_OK) return v;
        const DevParams d = dev_params(params[s], variant);
        tp += d.P;
        tb += d.B;
        tc += d.C;
    }
    if (tp + tb > (1L << 30) || tc > (1L << 30)) return K3DOM_ERR_CAPACITY;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return K3DOM_ERR_NO_DEVICE;
    if (device < 0 || device >= ndev) return K3DOM_ERR_INVALID_ARGUMENT;
    k3dom_handle* h = new (std::nothrow) k3dom_handle();
    if (!h) return K3DOM_ERR_OUT_OF_MEMORY;
    h->device = device;
    h->variant = variant;
    h->S = n_scenes;
    h->sc.resize(n_scenes);
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
    if ((e = sort_init()) || (e = onesweep_init()) || (e = evidence_init())) return bail(e);

    // scene ranges
    int P = 0, B = 0, C = 0;
    for (int s = 0; s < n_scenes; ++s) {
        SceneHost& x = h->sc[s];
        x.params = params[s];
        if (x.params.max_points <= 0) x.params.max_points = 131072;
        x.max_points = x.params.max_points;
        x.dp = dev_params(x.params, variant);
        h->off.part[s] = P;
        h->off.birth[s] = B;
        h->off.joint[s] = P + B;
        h->off.cell[s] = C;
        P += x.dp.P;
        B += x.dp.B;
        C += x.dp.C;
    }
    h->off.part[n_scenes] = P;
    h->off.birth[n_scenes] = B;
    h->off.joint[n_scenes] = P + B;
    h->off.cell[n_scenes] = C;
    h->P = P;
    h->B = B;
    h->C = C;

    // the frame's own stream at the highest priority: where the evidence kernel runs beside
    // prediction and assignment (on st3), the block scheduler hands freed SM slots to the
    // particle stages first, which the evidence waits for at the cell update
    int prio_low = 0, prio_high = 0;
    if ((e = cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high))) return bail(e);
    if ((e = cudaStreamCreateWithPriority(&h->st, cudaStreamNonBlocking, prio_high))) return bail(e);
    if ((e = cudaStreamCreateWithPriority(&h->st2, cudaStreamNonBlocking, prio_low))) return bail(e);
    if ((e = cudaStreamCreateWithPriority(&h->st3, cudaStreamNonBlocking, prio_low))) return bail(e);
    if ((e = cudaStreamCreateWithFlags(&h->st4, cudaStreamNonBlocking))) return bail(e);
    if ((e = cudaEventCreateWithFlags(&h->ev_out, cudaEventDisableTiming))) return bail(e);
    if ((e = cudaEventCreateWithFlags(&h->ev_out_done, cudaEventDisableTiming))) return bail(e);
    if ((e = cudaMallocHost((void**)&h->status_host, sizeof(DevStatus)))) return bail(e);
    std::memset(h->status_host, 0, sizeof(DevStatus));
    if ((e = cudaEventCreateWithFlags(&h->ev_bin, cudaEventDisableTiming))) return bail(e);
    if ((e = cudaEventCreateWithFlags(&h->ev_cells, cudaEventDisableTiming))) return bail(e);
    if ((e = cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming))) return bail(e);
    if ((e = cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming))) return bail(e);
    if ((e = cudaEventCreateWithFlags(&h->ev_staged, cudaEventDisableTiming))) return bail(e);
    if ((e = cudaEventRecord(h->ev_staged, h->st))) return bail(e);
    for (auto& ev : h->ev_t)
        if ((e = cudaEventCreate(&ev))) return bail(e);
    if ((e = cudaMallocHost((void**)&h->fp_host, sizeof(FrameParams) * n_scenes))) return bail(e);
    std::memset(h->fp_host, 0, sizeof(FrameParams) * n_scenes);
    if ((e = h->alloc(&h->fp_dev, n_scenes)) || (e = h->alloc(&h->status, 1)) ||
        (e = h->alloc(&h->sc_dev, n_scenes)) || (e = h->alloc(&h->off_dev, 1)))
        return bail(e);
    if ((e = h->alloc_particles(&h->A, P)) || (e = h->alloc_particles(&h->Ss, P)) ||
        (e = h->alloc_particles(&h->Bp, B)))
        return bail(e);
    if ((e = h->alloc(&h->X, 2 * (size_t)P))) return bail(e);
    if ((e = h->alloc(&h->sorted_keys, P)) || (e = h->alloc(&h->perm, P)) || (e = h->alloc(&h->alt_k, P)) ||
        (e = h->alloc(&h->alt_v, P)) || (e = h->alloc(&h->seg_rec, seg_rec_count(P))) ||
        (e = h->alloc(&h->res_br, res_bracket_count(P))))
        return bail(e);
    if ((e = h->alloc_cells(&h->cs[0], C)) || (e = h->alloc_cells(&h->cs[1], C))) return bail(e);
    CellWork& cw = h->cw;
    if ((e = h->alloc(&cw.start, C)) || (e = h->alloc(&cw.end, C)) || (e = h->alloc(&h->start2, C)) ||
        (e = h->alloc(&h->end2, C)) || (e = h->alloc(&cw.sum_w, C)) || (e = h->alloc(&cw.sum_wvx, C)) ||
        (e = h->alloc(&cw.sum_wvy, C)) || (e = h->alloc(&cw.sum_wvz, C)) || (e = h->alloc(&cw.factor, C)) ||
        (e = h->alloc(&cw.divisor, C)) || (e = h->alloc(&cw.meas_occ, C)) || (e = h->alloc(&cw.meas_free, C)) ||
        (e = h->alloc(&cw.del_occ, C)) || (e = h->alloc(&cw.del_free, C)))
        return bail(e);
    if ((e = h->alloc(&h->born_cum, C)) || (e = h->alloc(&h->joint_cum, (size_t)P + B)) ||
        (e = h->alloc(&h->joint_max, n_scenes)) || (e = h->alloc(&h->ancestors, P)))
        return bail(e);
    // exact-scan plans: born masses per scene; joint weights (persistent ++ births) per scene
    {
        std::vector<ExactTile> pb, pj;
        for (int s = 0; s < n_scenes; ++s) {
            const SceneHost& x = h->sc[s];
            float* in1[1] = {h->cs[0].born_m + h->off.cell[s]};
            const long n1[1] = {x.dp.C};
            exact_plan_add(pb, in1, n1, 1, h->born_cum + h->off.cell[s]);
            float* in2[2] = {h->Ss.w + h->off.part[s], h->Bp.w + h->off.birth[s]};
            const long n2[2] = {x.dp.P, x.dp.B};
            exact_plan_add(pj, in2, n2, 2, h->joint_cum + h->off.joint[s]);
        }
        h->plan_born_n = (int)pb.size();
        h->plan_joint_n = (int)pj.size();
        if ((e = h->alloc(&h->plan_born, pb.size())) || (e = h->alloc(&h->plan_joint, pj.size()))) return bail(e);
        if ((e = cudaMemcpyAsync(h->plan_born, pb.data(), sizeof(ExactTile) * pb.size(), cudaMemcpyHostToDevice,
                                 h->st)) ||
            (e = cudaMemcpyAsync(h->plan_joint, pj.data(), sizeof(ExactTile) * pj.size(), cudaMemcpyHostToDevice,
                                 h->st)) ||
            (e = cudaStreamSynchronize(h->st)))
            return bail(e);
        const size_t sb = exact_plan_scratch_bytes(std::max(h->plan_born_n, h->plan_joint_n));
        unsigned char* es = nullptr;
        if ((e = h->alloc(&es, sb))) return bail(e);
        h->exact_scratch = es;
    }
    if ((e = h->alloc(&h->draw_keys, P)) || (e = h->alloc(&h->draw_sorted, P)) || (e = h->alloc(&h->draw_alt, P)))
        return bail(e);
    // sort scratch of the particle sort, and a separate one for the draw sort (it runs
    // concurrently on the second stream; the draw keys carry the scene index above 24 bits)
    h->os_words = onesweep_scratch_words(P, key_bits_for(h->C));
    if ((e = h->alloc(&h->os_scratch, h->os_words))) return bail(e);
    h->os_draw_words = onesweep_scratch_words(P, draw_key_bits(h->S));
    if ((e = h->alloc(&h->os_draw, h->os_draw_words))) return bail(e);
    if ((e = alloc_ray_buffers(h))) return bail(e);
    // DOM_c::initialize (src/common/dom.cu:90-109): cells to priors
    launch_cells_init(h->batch(), h->cs[0], h->cw, h->st);
    launch_cells_init(h->batch(), h->cs[1], h->cw, h->st);
    if ((e = cudaGetLastError()) || (e = cudaStreamSynchronize(h->st))) return bail(e);
    *out = h;
    return K3DOM_OK;
}

k3dom_status k3dom_create(const k3dom_params* params, k3dom_variant variant, int device, k3dom_handle** out) {
    return k3dom_batch_create(params, 1, variant, device, out);
}

k3dom_status k3dom_destroy(k3dom_handle* h) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    cudaStreamSynchronize(h->st);
    cudaStreamSynchronize(h->st2);
    cudaStreamSynchronize(h->st3);
    cudaStreamSynchronize(h->st4);
    h->release();
    delete h;
    return K3DOM_OK;
}

k3dom_status k3dom_batch_size(k3dom_handle* h, int32_t* n_scenes) {
    if (!h || !n_scenes) return K3DOM_ERR_INVALID_ARGUMENT;
    *n_scenes = h->S;
    return K3DOM_OK;
}

k3dom_status k3dom_select_scene(k3dom_handle* h, int32_t scene) {
    if (!h || scene < 0 || scene >= h->S) return K3DOM_ERR_INVALID_ARGUMENT;
    h->cur = scene;
    return K3DOM_OK;
}

k3dom_status k3dom_batch_update_pose(k3dom_handle* h, int32_t scene, float x, float y, float z) {
    if (!h || scene < 0 || scene >= h->S) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    SceneHost& sh = h->sc[scene];
    const k3dom_params& p = sh.params;
    sh.sensor_pos[0] = x;
    sh.sensor_pos[1] = y;
    sh.sensor_pos[2] = z;
    if (!sh.first_pose_received) {
        sh.first_pose_received = true;
        sh.center_pos[0] = x - p.sensor_off_x;
        sh.center_pos[1] = y - p.sensor_off_y;
        sh.center_pos[2] = z - p.sensor_off_z;
        return K3DOM_OK;
    }
    const int mx = static_cast<int>((x - sh.center_pos[0] - p.sensor_off_x) / p.resolution);
    const int my = static_cast<int>((y - sh.center_pos[1] - p.sensor_off_y) / p.resolution);
    const int mz = static_cast<int>((z - sh.center_pos[2] - p.sensor_off_z) / p.resolution);
    if (std::abs(mx) >= p.map_shift_thresh || std::abs(my) >= p.map_shift_thresh ||
        std::abs(mz) >= p.map_shift_thresh) {
        cudaError_t e;
        const long co = h->off.cell[scene];
        if (sh.shift_pending) {
            // a second shift before any prediction: apply the first to the particles now so
            // each subtraction rounds exactly as moveParticlesKernel's would
            if ((e = ensure_a_current(h))) return h->fail(e);
            h->x_current = false;
            launch_shift_particles(sh.dp.P, offset_particles(h->A, h->off.part[scene]), sh.pending_shift[0],
                                   sh.pending_shift[1], sh.pending_shift[2], h->st);
        }
        // shift into the spare buffers, then copy back so every captured pointer stays valid
        launch_map_shift_full(sh.dp, offset_cells(h->cs[0], co), offset_cells(h->cs[1], co), h->cw.start + co,
                              h->cw.end + co, h->start2 + co, h->end2 + co, mx, my, mz, h->st);
        if ((e = copy_cells_back(h, scene))) return h->fail(e);
        sh.shift_pending = true;
        sh.pending_shift[0] = mx;
        sh.pending_shift[1] = my;
        sh.pending_shift[2] = mz;
        if ((e = cudaGetLastError())) return h->fail(e);
        sh.center_pos[0] += mx * p.resolution;
        sh.center_pos[1] += my * p.resolution;
        sh.center_pos[2] += mz * p.resolution;
    }
    return K3DOM_OK;
}

k3dom_status k3dom_set_point_transform(k3dom_handle* h, int32_t scene, const float* rotation, const float* translation) {
    if (!h || scene < 0 || scene >= h->S) return K3DOM_ERR_INVALID_ARGUMENT;
    SceneHost& x = h->sc[scene];
    if (!rotation) {
        x.has_transform = false;
        return K3DOM_OK;
    }
    for (int i = 0; i < 9; ++i)
        if (!std::isfinite(rotation[i])) return K3DOM_ERR_INVALID_INPUT;
    if (translation)
        for (int i = 0; i < 3; ++i)
            if (!std::isfinite(translation[i])) return K3DOM_ERR_INVALID_INPUT;
    std::memcpy(x.rot, rotation, sizeof(x.rot));
    for (int i = 0; i < 3; ++i) x.trans[i] = translation ? translation[i] : 0.0f;
    x.has_transform = true;
    return K3DOM_OK;
}

k3dom_status k3dom_update_pose(k3dom_handle* h, float x, float y, float z) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    return k3dom_batch_update_pose(h, h->cur, x, y, z);
}

static cudaError_t copy_cells_back(k3dom_handle* h, int s) {
    const long co = h->off.cell[s];
    const size_t b = sizeof(float) * (size_t)h->sc[s].dp.C;
    const CellState src = offset_cells(h->cs[1], co);
    const CellState dst = offset_cells(h->cs[0], co);
    const float* from[] = {src.free_m, src.static_m, src.dyn_m, src.occ_m, src.pers_m,
                           src.pred_m, src.born_m,   src.mvx,   src.mvy,   src.mvz};
    float* to[] = {dst.free_m, dst.static_m, dst.dyn_m, dst.occ_m, dst.pers_m,
                   dst.pred_m, dst.born_m,   dst.mvx,   dst.mvy,   dst.mvz};
    cudaError_t e;
    for (int i = 0; i < 10; ++i)
        if ((e = cudaMemcpyAsync(to[i], from[i], b, cudaMemcpyDeviceToDevice, h->st))) return e;
    const size_t bi = sizeof(int) * (size_t)h->sc[s].dp.C;
    if ((e = cudaMemcpyAsync(h->cw.start + co, h->start2 + co, bi, cudaMemcpyDeviceToDevice, h->st))) return e;
    return cudaMemcpyAsync(h->cw.end + co, h->end2 + co, bi, cudaMemcpyDeviceToDevice, h->st);
}

static k3dom_status finish_sync(k3dom_handle* h) {
    cudaError_t e = cudaSuccess;
    if (h->status) e = cudaMemcpyAsync(h->status_host, h->status, sizeof(DevStatus), cudaMemcpyDeviceToHost, h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
    if (e != cudaSuccess) return h->fail(e);
    if (h->status && (h->status_host->sort_timeout || h->status_host->copy_timeout)) {
        // a bounded device wait gave up (the particle sort's look-back, or a bulk copy of the
        // cell update): its output is incomplete; report it once
        h->status_host->sort_timeout = h->status_host->copy_timeout = 0;
        e = cudaMemsetAsync(&h->status->sort_timeout, 0, 2 * sizeof(unsigned int), h->st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->st);
        if (e != cudaSuccess) return h->fail(e);
        return K3DOM_ERR_TIMEOUT;
    }
    if (h->status && h->status_host->overflow) return K3DOM_ERR_CAPACITY;
    return K3DOM_OK;
}

// One frame of every scene: t[s], points (xs[s], ys[s], zs[s], n[s]).
static k3dom_status update_impl(k3dom_handle* h, const float* t, const float* const* xs, const float* const* ys,
                                const float* const* zs, const int32_t* n, k3dom_mem mem, bool sync) {
    if (!h || !t || !n || !xs) return K3DOM_ERR_INVALID_ARGUMENT;
    const int S = h->S;
    for (int s = 0; s < S; ++s) {
        k3dom_status c = check_points(xs[s], ys ? ys[s] : nullptr, zs ? zs[s] : nullptr, n[s], mem);
        if (c != K3DOM_OK) return c;
    }
    // scenes step together: the first frame initialises every scene (src/k3dom/dom.cu:32)
    const bool steady = h->sc[0].updated_time > 0.0f;
    for (int s = 1; s < S; ++s)
        if ((h->sc[s].updated_time > 0.0f) != steady) return K3DOM_ERR_NOT_READY;
    cudaSetDevice(h->device);
    k3dom_status st = grow_points(h, n);
    if (st != K3DOM_OK) return st;
    std::vector<float> dt(S);
    std::vector<int> np(S);
    for (int s = 0; s < S; ++s) {
        dt[s] = steady ? t[s] - h->sc[s].updated_time : 0.0f;
        np[s] = n[s];
    }
    if ((st = set_frame_params(h, dt.data(), np.data())) != K3DOM_OK) return st;
    const long l_up = g_launches;
    if ((st = upload_all(h, xs, ys, zs, n, mem, sync, true)) != K3DOM_OK) return st;
    h->launches_upload = (int)(g_launches - l_up);
    cudaError_t e;
    bool timed = false;
    if (steady) {
        const bool tuning = h->tune_next >= 0;
        if (tuning) {
            const int k = h->tune_next;
            if ((e = apply_tuning(h, k % kRuleCount, kTuneChunks[k / kRuleCount]))) return h->fail(e);
            // the candidate's upload of this frame's points happened before any re-layout
            // changed the point slots: stage them again
            if ((st = set_frame_params(h, dt.data(), np.data())) != K3DOM_OK) return st;
            if ((st = upload_all(h, xs, ys, zs, n, mem, sync, false)) != K3DOM_OK) return st;
        }
        if (h->timing || !h->graph_mode || tuning) {
            const bool was = h->timing;
            h->timing = true;
            e = enq_frame(h);
            h->timing = was;
            if (e) return h->fail(e);
            timed = true;
        } else {
            if (!h->graph_exec) {
                if ((e = cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal))) return h->fail(e);
                cudaError_t ce = enq_frame(h);
                cudaGraph_t g = nullptr;
                e = cudaStreamEndCapture(h->st, &g);
                if (ce != cudaSuccess) {
                    if (g) cudaGraphDestroy(g);
                    return h->fail(ce);
                }
                if (e != cudaSuccess) return h->fail(e);
                h->graph = g;
                // the kernels keep their streams' priorities inside the graph
                if ((e = cudaGraphInstantiate(&h->graph_exec, g, cudaGraphInstantiateFlagUseNodePriority)))
                    return h->fail(e);
            }
            if ((e = cudaGraphLaunch(h->graph_exec, h->st))) return h->fail(e);
        }
        h->births_done = true;
    } else {
        // DOM::initializeParticles (src/k3dom/dom.cu:52-77; src/dsphdmib/dom.cu:55-82)
        if ((e = enq_occupancy(h, true))) return h->fail(e);
        if ((e = enq_init_particles(h))) return h->fail(e);
        if ((e = enq_output(h)) || (e = enq_output_join(h))) return h->fail(e);
    }
    for (int s = 0; s < S; ++s) {
        SceneHost& x = h->sc[s];
        x.shift_pending = false;
        x.pending_shift[0] = x.pending_shift[1] = x.pending_shift[2] = 0;
        x.updated_time = t[s];
        x.frame += 1;
        if (h->ds()) x.iteration += 1;  // src/dsphdmib/dom.cu:52
        x.initialized = true;
    }
    if (!sync && !timed) return K3DOM_OK;
    st = finish_sync(h);
    if (st != K3DOM_OK || !timed) return st;
    read_times(h);
    if (h->tune_next >= 0) {
        // the evidence stage (ray lists + evidence kernels) decides between candidates
        const float ms = h->times.occupancy_ms;
        h->tune_ms[h->tune_next] = ms;
        if (h->tune_next == 0 || ms < h->tune_best_ms) {
            h->tune_best_ms = ms;
            h->tune_best = h->tune_next;
        }
        h->tune_next += 1;
        if (h->tune_next >= kTuneCount) {
            h->tune_next = -1;
            h->tuned = 1;
            if ((e = apply_tuning(h, h->tune_best % kRuleCount, kTuneChunks[h->tune_best / kRuleCount])))
                return h->fail(e);
        }
    }
    return K3DOM_OK;
}

k3dom_status k3dom_batch_update(k3dom_handle* h, const float* t, const float* const* xs, const float* const* ys,
                                const float* const* zs, const int32_t* n, k3dom_mem mem) {
    return update_impl(h, t, xs, ys, zs, n, mem, true);
}

k3dom_status k3dom_batch_update_async(k3dom_handle* h, const float* t, const float* const* xs,
                                      const float* const* ys, const float* const* zs, const int32_t* n,
                                      k3dom_mem mem) {
    return update_impl(h, t, xs, ys, zs, n, mem, false);
}

k3dom_status k3dom_update_grid(k3dom_handle* h, float t, const float* xs, const float* ys, const float* zs, int32_t n,
                               k3dom_mem mem) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    if (h->S != 1) return K3DOM_ERR_INVALID_ARGUMENT;
    return update_impl(h, &t, &xs, &ys, &zs, &n, mem, true);
}

k3dom_status k3dom_update_grid_async(k3dom_handle* h, float t, const float* xs, const float* ys, const float* zs,
                                     int32_t n, k3dom_mem mem) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    if (h->S != 1) return K3DOM_ERR_INVALID_ARGUMENT;
    return update_impl(h, &t, &xs, &ys, &zs, &n, mem, false);
}

k3dom_status k3dom_synchronize(k3dom_handle* h) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    k3dom_status s = finish_sync(h);
    if (s == K3DOM_OK && h->timing) read_times(h);
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

// ---- evidence tuning
k3dom_status k3dom_autotune(k3dom_handle* h, int enabled) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    if (enabled) {
        h->tune_next = 0;
        h->tuned = 0;
        h->tune_ms.assign(kTuneCount, 0.0f);
    } else {
        h->tune_next = -1;
    }
    return K3DOM_OK;
}

k3dom_status k3dom_get_tuning(k3dom_handle* h, k3dom_tuning* out) {
    if (!h || !out) return K3DOM_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    out->tile_rule = h->tile_rule;
    out->chunk = h->chunk;
    out->tuned = h->tuned;
    out->tuning = h->tune_next >= 0 ? 1 : 0;
    out->candidates = kTuneCount;
    out->best_ms = h->tune_best_ms;
    for (int k = 0; k < kTuneCount && k < (int)h->tune_ms.size() && k < K3DOM_TUNE_MAX_CANDIDATES; ++k)
        out->candidate_ms[k] = h->tune_ms[k];
    if (h->ds()) {
        k3dom_ds_evidence_blocks(&out->evidence_count_blocks, &out->evidence_blocks);
    } else {
        out->evidence_blocks = k3dom_evidence_blocks(h->rb.chunk);
        out->evidence_count_blocks = 0;
    }
    return K3DOM_OK;
}

k3dom_status k3dom_set_sort_wait(k3dom_handle* h, uint32_t max_polls, int32_t skip_tile) {
    if (!h || skip_tile < -1) return K3DOM_ERR_INVALID_ARGUMENT;
    h->sort_wait.max_polls = max_polls;
    h->sort_wait.skip_tile = skip_tile;
    h->drop_graph();  // the captured frame holds the old arguments
    return K3DOM_OK;
}

k3dom_status k3dom_set_tuning(k3dom_handle* h, int32_t tile_rule, int32_t chunk) {
    if (!h || tile_rule < 0 || tile_rule >= kRuleCount || chunk < 32 || chunk > 1024) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    h->tune_next = -1;
    cudaError_t e = apply_tuning(h, tile_rule, chunk);
    return e == cudaSuccess ? K3DOM_OK : h->fail(e);
}

// ---- stage calls (all scenes; the point-taking calls need a single scene)
#define STAGE_BEGIN                          \
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT; \
    cudaSetDevice(h->device);                \
    cudaError_t e;

static void clear_shifts(k3dom_handle* h) {
    for (auto& x : h->sc) {
        x.shift_pending = false;
        x.pending_shift[0] = x.pending_shift[1] = x.pending_shift[2] = 0;
    }
}

k3dom_status k3dom_particle_prediction(k3dom_handle* h, float dt) {
    STAGE_BEGIN
    k3dom_status s = set_frame_params_all(h, dt, 0);
    if (s != K3DOM_OK) return s;
    if ((e = enq_predict(h))) return h->fail(e);
    clear_shifts(h);
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
    if (h->S != 1) return K3DOM_ERR_INVALID_ARGUMENT;
    k3dom_status s = check_points(xs, ys, zs, n, mem);
    if (s != K3DOM_OK) return s;
    if ((s = grow_points(h, &n)) != K3DOM_OK) return s;
    if ((s = set_frame_params_all(h, dt, n)) != K3DOM_OK) return s;
    if ((s = upload_all(h, &xs, &ys, &zs, &n, mem, false, true)) != K3DOM_OK) return s;
    if ((e = enq_occupancy(h, false))) return h->fail(e);
    return finish_sync(h);
}

k3dom_status k3dom_update_persistent_particles(k3dom_handle* h) {
    STAGE_BEGIN
    if ((e = enq_persistent(h, h->st))) return h->fail(e);
    return finish_sync(h);
}

k3dom_status k3dom_initialize_new_particles(k3dom_handle* h) {
    STAGE_BEGIN
    k3dom_status s = set_frame_params_all(h, h->fp_host[0].dt, h->fp_host[0].n_points);
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
    k3dom_status s = set_frame_params_all(h, h->fp_host[0].dt, h->fp_host[0].n_points);
    if (s != K3DOM_OK) return s;
    if ((e = enq_resample(h, false))) return h->fail(e);
    return finish_sync(h);
}

k3dom_status k3dom_initialize_particles(k3dom_handle* h, const float* xs, const float* ys, const float* zs, int32_t n,
                                        k3dom_mem mem) {
    STAGE_BEGIN
    if (h->S != 1) return K3DOM_ERR_INVALID_ARGUMENT;
    k3dom_status s = check_points(xs, ys, zs, n, mem);
    if (s != K3DOM_OK) return s;
    if ((s = grow_points(h, &n)) != K3DOM_OK) return s;
    if ((s = set_frame_params_all(h, 0.0f, n)) != K3DOM_OK) return s;
    if ((s = upload_all(h, &xs, &ys, &zs, &n, mem, false, true)) != K3DOM_OK) return s;
    if ((e = enq_occupancy(h, true))) return h->fail(e);
    if ((e = enq_init_particles(h))) return h->fail(e);
    return finish_sync(h);
}

k3dom_status k3dom_finish_frame(k3dom_handle* h, float t) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    for (auto& x : h->sc) {
        x.updated_time = t;
        x.frame += 1;
        if (h->ds()) x.iteration += 1;
        x.initialized = true;
    }
    return K3DOM_OK;
}

k3dom_status k3dom_set_frame_index(k3dom_handle* h, int32_t frame) {
    if (!h || frame < 0) return K3DOM_ERR_INVALID_ARGUMENT;
    for (auto& x : h->sc) x.frame = (uint32_t)frame;
    return K3DOM_OK;
}

// ---- info (selected scene)
k3dom_status k3dom_get_info(k3dom_handle* h, k3dom_info* o) {
    if (!h || !o) return K3DOM_ERR_INVALID_ARGUMENT;
    const SceneHost& x = h->sc[h->cur];
    o->grid_size = x.dp.G;
    o->grid_size_z = x.dp.Gz;
    o->grid_cell_count = x.dp.C;
    o->particle_count = x.dp.P;
    o->new_born_particle_count = x.dp.B;
    o->iteration = x.iteration;
    o->variant = (int)h->variant;
    o->initialized = x.initialized ? 1 : 0;
    o->resolution = x.params.resolution;
    o->center_x = x.center_pos[0];
    o->center_y = x.center_pos[1];
    o->center_z = x.center_pos[2];
    o->sensor_x = x.sensor_pos[0];
    o->sensor_y = x.sensor_pos[1];
    o->sensor_z = x.sensor_pos[2];
    o->updated_time = x.updated_time;
    o->max_points = x.max_points;
    o->frame_index = (int32_t)x.frame;
    return K3DOM_OK;
}

k3dom_status k3dom_index_to_coord(k3dom_handle* h, int32_t i, float* x, float* y, float* z) {
    // DOM_c::indexToCoordX/Y/Z (include/common/dom.h:70-81)
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    const SceneHost& s = h->sc[h->cur];
    if (i < 0 || i >= s.dp.C) return K3DOM_ERR_INVALID_ARGUMENT;
    const int G = s.dp.G;
    const float r = s.params.resolution;
    if (x) *x = (i % G + 0.5f) * r - s.params.size / 2.0f + s.center_pos[0];
    if (y) *y = ((i % (G * G)) / G + 0.5f) * r - s.params.size / 2.0f + s.center_pos[1];
    if (z) *z = (i / (G * G) + 0.5f) * r - s.params.size_z / 2.0f + s.center_pos[2];
    return K3DOM_OK;
}

// ---- readback (selected scene)
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

// dst[i] = src[i] - base where src[i] >= 0 (global -> scene-local indices); weights: |w|.
__global__ void k_rebase(const int* __restrict__ src, int* __restrict__ dst, int n, int base, int keep_neg) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int v = src[i];
    dst[i] = (keep_neg && v < 0) ? v : v - base;
}

// strips the penalty flag (sign bit) kept in the sorted and birth weights between stages
__global__ void k_abs_copy(const float* __restrict__ src, float* __restrict__ dst, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = fabsf(src[i]);
}

static k3dom_status deliver_rebased(k3dom_handle* h, int32_t* dst, const int* src, int n, int base, bool keep_neg,
                                    k3dom_mem mem) {
    k3dom_status s = ensure_export(h, sizeof(int) * (size_t)std::max(n, 1));
    if (s != K3DOM_OK) return s;
    ++g_launches;
    k_rebase<<<div_up(std::max(n, 1), 256), 256, 0, h->st>>>(src, (int*)h->export_buf, n, base, keep_neg ? 1 : 0);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return h->fail(e);
    return deliver(h, dst, h->export_buf, sizeof(int) * (size_t)n, mem);
}

k3dom_status k3dom_get_cell_field(k3dom_handle* h, k3dom_cell_field field, float* dst, k3dom_mem mem) {
    if (!h || !dst || (int)field < 0 || field >= K3DOM_CELL_FIELD_COUNT) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    const int s = h->cur;
    const SceneHost& x = h->sc[s];
    const long co = h->off.cell[s];
    const size_t bytes = sizeof(float) * (size_t)x.dp.C;
    float* out = dst;
    if (mem == K3DOM_MEM_HOST) {
        k3dom_status r = ensure_export(h, bytes);
        if (r != K3DOM_OK) return r;
        out = (float*)h->export_buf;
    }
    launch_export_field(x.dp, (int)field, offset_cells(h->cells(), co), offset_work(h->cw, co),
                        h->births_done ? h->born_cum + co : nullptr, h->off.part[s], out, h->st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return h->fail(e);
    if (mem == K3DOM_MEM_HOST) return deliver(h, dst, out, bytes, mem);
    e = cudaStreamSynchronize(h->st);
    return e == cudaSuccess ? K3DOM_OK : h->fail(e);
}

k3dom_status k3dom_set_output(k3dom_handle* h, k3dom_cell_field field, float* dst, k3dom_mem mem) {
    if (!h || (dst && ((int)field < 0 || field >= K3DOM_CELL_FIELD_COUNT))) return K3DOM_ERR_INVALID_ARGUMENT;
    if (dst && mem == K3DOM_MEM_HOST && !is_pinned_host(dst)) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    cudaError_t e = cudaStreamSynchronize(h->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->st4);
    if (e != cudaSuccess) return h->fail(e);
    // device staging for a host destination: sized for every cell of the handle, so any scene fits
    if (dst && mem == K3DOM_MEM_HOST && !h->out_buf &&
        (e = cudaMalloc((void**)&h->out_buf, sizeof(float) * (size_t)std::max(h->C, 1))))
        return h->fail(e);
    h->out_field = dst ? (int)field : -1;
    h->out_dst = dst;
    h->out_mem = mem;
    h->out_scene = h->cur;
    h->drop_graph();  // the frame graph holds the export: capture it again
    return K3DOM_OK;
}

k3dom_status k3dom_get_cell_ranges(k3dom_handle* h, int32_t* start, int32_t* end, k3dom_mem mem) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    const int s = h->cur;
    const long co = h->off.cell[s];
    const int C = h->sc[s].dp.C, base = h->off.part[s];
    k3dom_status r = K3DOM_OK;
    if (start) r = deliver_rebased(h, start, h->cw.start + co, C, base, true, mem);
    if (r == K3DOM_OK && end) r = deliver_rebased(h, end, h->cw.end + co, C, base, true, mem);
    return r;
}

k3dom_status k3dom_get_gridcell_aos(k3dom_handle* h, void* dst, k3dom_mem mem) {
    if (!h || !dst) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    const int s = h->cur;
    const SceneHost& x = h->sc[s];
    const long co = h->off.cell[s];
    const size_t bytes = (size_t)K3DOM_GRIDCELL_BYTES * x.dp.C;
    void* out = dst;
    if (mem == K3DOM_MEM_HOST) {
        k3dom_status r = ensure_export(h, bytes);
        if (r != K3DOM_OK) return r;
        out = h->export_buf;
    }
    launch_export_gridcell(x.dp, offset_cells(h->cells(), co), offset_work(h->cw, co),
                           h->births_done ? h->born_cum + co : nullptr, h->off.part[s], out, h->st);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return h->fail(e);
    if (mem == K3DOM_MEM_HOST) return deliver(h, dst, out, bytes, mem);
    e = cudaStreamSynchronize(h->st);
    return e == cudaSuccess ? K3DOM_OK : h->fail(e);
}

k3dom_status k3dom_get_mappoints(k3dom_handle* h, float* dst, k3dom_mem mem) {
    if (!h || !dst) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    const int s = h->cur;
    const SceneHost& x = h->sc[s];
    const long co = h->off.cell[s];
    const size_t bytes = sizeof(float) * K3DOM_MAPPOINT_FLOATS * (size_t)x.dp.C;
    float* out = dst;
    if (mem == K3DOM_MEM_HOST) {
        k3dom_status r = ensure_export(h, bytes);
        if (r != K3DOM_OK) return r;
        out = (float*)h->export_buf;
    }
    launch_export_mappoints(x.dp, x.center_pos[0], x.center_pos[1], x.center_pos[2], offset_cells(h->cells(), co),
                            offset_work(h->cw, co), out, h->st);
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
    const long co = h->off.cell[h->cur];
    const size_t bytes = sizeof(float) * (size_t)h->sc[h->cur].dp.C;
    const cudaMemcpyKind k = mem == K3DOM_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    const CellState c = offset_cells(h->cells(), co);
    cudaError_t e;
    if (f && (e = cudaMemcpyAsync(c.free_m, f, bytes, k, h->st))) return h->fail(e);
    if (s && (e = cudaMemcpyAsync(c.static_m, s, bytes, k, h->st))) return h->fail(e);
    if (d && (e = cudaMemcpyAsync(c.dyn_m, d, bytes, k, h->st))) return h->fail(e);
    if (o && (e = cudaMemcpyAsync(c.occ_m, o, bytes, k, h->st))) return h->fail(e);
    e = cudaStreamSynchronize(h->st);
    return e == cudaSuccess ? K3DOM_OK : h->fail(e);
}

static bool pick_set(k3dom_handle* h, k3dom_particle_set set, Particles* q, int* n) {
    const int s = h->cur;
    switch (set) {
        case K3DOM_PARTICLES_PERSISTENT: *n = h->sc[s].dp.P; *q = offset_particles(h->A, h->off.part[s]); return true;
        case K3DOM_PARTICLES_SORTED: *n = h->sc[s].dp.P; *q = offset_particles(h->Ss, h->off.part[s]); return true;
        case K3DOM_PARTICLES_BIRTH: *n = h->sc[s].dp.B; *q = offset_particles(h->Bp, h->off.birth[s]); return true;
    }
    return false;
}

k3dom_status k3dom_get_particles(k3dom_handle* h, k3dom_particle_set set, float* pos, float* vel, float* weight,
                                 int32_t* cell_idx, uint8_t* associated, k3dom_mem mem) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    int n = 0;
    Particles q;
    if (!pick_set(h, set, &q, &n)) return K3DOM_ERR_INVALID_ARGUMENT;
    const cudaMemcpyKind k = mem == K3DOM_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    cudaError_t e;
    if (set == K3DOM_PARTICLES_PERSISTENT && (e = ensure_a_current(h))) return h->fail(e);
    auto strided = [&](float* dst, const float* a, const float* b, const float* c) -> cudaError_t {
        cudaError_t r;
        if ((r = cudaMemcpy2DAsync(dst, 3 * sizeof(float), a, sizeof(float), sizeof(float), n, k, h->st))) return r;
        if ((r = cudaMemcpy2DAsync(dst + 1, 3 * sizeof(float), b, sizeof(float), sizeof(float), n, k, h->st))) return r;
        return cudaMemcpy2DAsync(dst + 2, 3 * sizeof(float), c, sizeof(float), sizeof(float), n, k, h->st);
    };
    if (pos && (e = strided(pos, q.px, q.py, q.pz))) return h->fail(e);
    if (vel && (e = strided(vel, q.vx, q.vy, q.vz))) return h->fail(e);
    if (weight) {
        k3dom_status s = ensure_export(h, sizeof(float) * (size_t)n);
        if (s != K3DOM_OK) return s;
        ++g_launches;
        k_abs_copy<<<div_up(n, 256), 256, 0, h->st>>>(q.w, (float*)h->export_buf, n);
        if ((e = cudaMemcpyAsync(weight, h->export_buf, sizeof(float) * (size_t)n, k, h->st))) return h->fail(e);
        if ((e = cudaStreamSynchronize(h->st))) return h->fail(e);
    }
    if (cell_idx) {
        k3dom_status s = deliver_rebased(h, cell_idx, q.cell, n, h->off.cell[h->cur], false, mem);
        if (s != K3DOM_OK) return s;
    }
    if (associated && (e = cudaMemcpyAsync(associated, q.assoc, (size_t)n, k, h->st))) return h->fail(e);
    e = cudaStreamSynchronize(h->st);
    return e == cudaSuccess ? K3DOM_OK : h->fail(e);
}

__global__ void k_iota(uint32_t* a, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = (uint32_t)i;
}

__global__ void k_add_base(int* a, int n, int base) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] += base;
}

k3dom_status k3dom_set_particles(k3dom_handle* h, k3dom_particle_set set, const float* pos, const float* vel,
                                 const float* weight, const int32_t* cell_idx, const uint8_t* associated,
                                 k3dom_mem mem) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    int n = 0;
    Particles q;
    if (!pick_set(h, set, &q, &n)) return K3DOM_ERR_INVALID_ARGUMENT;
    if (set == K3DOM_PARTICLES_SORTED && (!cell_idx || h->S != 1)) return K3DOM_ERR_INVALID_ARGUMENT;
    const cudaMemcpyKind k = mem == K3DOM_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    cudaError_t e;
    // the fields not given keep their values: make A hold the whole current set first
    if ((e = ensure_a_current(h))) return h->fail(e);
    if (set == K3DOM_PARTICLES_PERSISTENT) h->x_current = false;
    auto strided = [&](const float* src, float* a, float* b, float* c) -> cudaError_t {
        cudaError_t r;
        if ((r = cudaMemcpy2DAsync(a, sizeof(float), src, 3 * sizeof(float), sizeof(float), n, k, h->st))) return r;
        if ((r = cudaMemcpy2DAsync(b, sizeof(float), src + 1, 3 * sizeof(float), sizeof(float), n, k, h->st))) return r;
        return cudaMemcpy2DAsync(c, sizeof(float), src + 2, 3 * sizeof(float), sizeof(float), n, k, h->st);
    };
    if (pos && (e = strided(pos, q.px, q.py, q.pz))) return h->fail(e);
    if (vel && (e = strided(vel, q.vx, q.vy, q.vz))) return h->fail(e);
    if (weight && (e = cudaMemcpyAsync(q.w, weight, sizeof(float) * (size_t)n, k, h->st))) return h->fail(e);
    if (cell_idx) {
        if ((e = cudaMemcpyAsync(q.cell, cell_idx, sizeof(int) * (size_t)n, k, h->st))) return h->fail(e);
        const int base = h->off.cell[h->cur];
        if (base != 0) {
            ++g_launches;
            k_add_base<<<div_up(n, 256), 256, 0, h->st>>>(q.cell, n, base);
        }
    }
    if (associated && (e = cudaMemcpyAsync(q.assoc, associated, (size_t)n, k, h->st))) return h->fail(e);
    if (set == K3DOM_PARTICLES_SORTED) {
        // a sorted set defines the cell ranges and sums: rebuild them from it in place
        if ((e = cudaMemcpyAsync(h->sorted_keys, q.cell, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, h->st)))
            return h->fail(e);
        ++g_launches;
        k_iota<<<div_up(n, 256), 256, 0, h->st>>>(h->perm, n);
        if ((e = cudaMemsetAsync(h->cw.start, 0xFF, sizeof(int) * (size_t)h->C, h->st))) return h->fail(e);
        if ((e = cudaMemsetAsync(h->cw.end, 0xFF, sizeof(int) * (size_t)h->C, h->st))) return h->fail(e);
        // the gather reads records: pack the sorted set into X (A holds the persistent set)
        launch_pack_records(n, h->Ss, h->X, h->st);
        h->x_current = false;
        launch_gather_segsum(h->batch(), h->X, h->Ss, h->sorted_keys, h->perm, h->cw, h->seg_rec, h->st);
    }
    e = cudaStreamSynchronize(h->st);
    return e == cudaSuccess ? K3DOM_OK : h->fail(e);
}

k3dom_status k3dom_get_sort_permutation(k3dom_handle* h, int32_t* perm, k3dom_mem mem) {
    if (!h || !perm) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    const int s = h->cur;
    return deliver_rebased(h, perm, reinterpret_cast<const int*>(h->perm) + h->off.part[s], h->sc[s].dp.P,
                           h->off.part[s], false, mem);
}

k3dom_status k3dom_get_ancestors(k3dom_handle* h, int32_t* anc, k3dom_mem mem) {
    if (!h || !anc) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    const int s = h->cur;
    return deliver(h, anc, h->ancestors + h->off.part[s], sizeof(int) * (size_t)h->sc[s].dp.P, mem);
}

k3dom_status k3dom_get_resampling_state(k3dom_handle* h, float* joint_cum, float* born_cum, float* joint_max,
                                        k3dom_mem mem) {
    if (!h) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(h->device);
    const int s = h->cur;
    const SceneHost& x = h->sc[s];
    k3dom_status r = K3DOM_OK;
    if (joint_cum)
        r = deliver(h, joint_cum, h->joint_cum + h->off.joint[s], sizeof(float) * ((size_t)x.dp.P + x.dp.B), mem);
    if (r == K3DOM_OK && born_cum)
        r = deliver(h, born_cum, h->born_cum + h->off.cell[s], sizeof(float) * (size_t)x.dp.C, mem);
    if (r == K3DOM_OK && joint_max) r = deliver(h, joint_max, h->joint_max + s, sizeof(float), mem);
    return r;
}

k3dom_status k3dom_debug_draws(uint64_t seed, int32_t frame, int32_t stage, int64_t first, int64_t count, float* dst,
                               k3dom_mem mem) {
    if (!dst || count < 0 || first < 0 || stage < 1 || stage > 4) return K3DOM_ERR_INVALID_ARGUMENT;
    const int per = stage == 1 ? 6 : (stage == 4 ? 1 : 3);
    const size_t bytes = sizeof(float) * (size_t)count * per;
    float* out = dst;
    cudaError_t e;
    if (mem == K3DOM_MEM_HOST) {
        if ((e = cudaMalloc((void**)&out, std::max<size_t>(bytes, 4))))
            return e == cudaErrorMemoryAllocation ? K3DOM_ERR_OUT_OF_MEMORY : K3DOM_ERR_CUDA;
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
    out->nonfinite_points = (int64_t)st.nonfinite_frame;
    out->ray_list_entries = (int64_t)st.ray_entries;
    out->ray_list_capacity = h->rb.capacity;
    out->work_items = (int64_t)st.work_items;
    out->overflow = (int32_t)st.overflow;
    out->kernel_launches_per_frame = h->launches_per_frame + h->launches_upload;
    out->kernel_evaluations = (int64_t)st.kernel_evals;
    return K3DOM_OK;
}

}  // extern "C"
