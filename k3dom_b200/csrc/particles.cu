// particles.cu -- particle-side kernels of the K3DOM frame: prediction (with the ego-motion
// particle shift folded in), the post-sort gather with per-cell segmented sums, the
// persistent reweight, first-frame initialisation, births and resampling.
//
// All float arithmetic that decides an integer result (positions -> voxel indices, velocity
// draws, birth slot and ancestor searches) is written with _rn intrinsics in the operation
// order of the reference, so it is not contracted into FMAs and reproduces the reference
// built with -fmad=false bit for bit.
#include <cuda_runtime.h>

#include "common.cuh"
#include "internal.h"

namespace k3dom {

using namespace k3dom_draws;

// ---------------------------------------------------------------- prediction
// predictKernel (src/common/kernel/predict.cu:12-59), preceded by moveParticlesKernel
// (src/common/kernel/ego_motion_compensation.cu:12-18) when a map shift is pending. Over all
// scenes of the batch; the Philox item is the particle's index within its scene and the
// stored cell index is the global one (scene cell offset + x + G y + G^2 z).
// One particle per thread (no grid-stride loop): every particle's loads are independent of
// another's stores, so the scheduler keeps many more of them in flight.
// The predicted particle goes out as one 32-byte record (x[2i] = px py pz vx, x[2i+1] = vy vz w
// assoc) plus its cell index in a.cell: the assignment then gathers each particle in one sector
// through the sort permutation, which jumps by several voxels' worth of particles.
__global__ void __launch_bounds__(kBlock) k_predict(Batch bt, Particles a, float4* __restrict__ x) {
    {
        const int i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= bt.P) return;
        const int sc = scene_of(bt.off->part, bt.S, i);
        const DevParams& p = bt.sc[sc].p;
        const FrameParams fp = bt.fp[sc];
        const int local = i - bt.off->part[sc];
        float px = a.px[i], py = a.py[i], pz = a.pz[i];
        float vx = a.vx[i], vy = a.vy[i], vz = a.vz[i];
        float w = a.w[i];
        if (fp.shift_pending) {
            px = __fsub_rn(px, (float)fp.shift_x);
            py = __fsub_rn(py, (float)fp.shift_y);
            pz = __fsub_rn(pz, (float)fp.shift_z);
        }
        float n[6];
        predict_normals(fp.seed, fp.frame, (uint64_t)local, n);
        const float noise_pos = p.noise_pos, noise_vel = p.noise_vel;
        // curand_normal(state, 0, s) = z * s + 0 (include/common/cuda_utils.h:33-35)
        const float npx = __fadd_rn(__fmul_rn(n[0], noise_pos), 0.0f);
        const float npy = __fadd_rn(__fmul_rn(n[1], noise_pos), 0.0f);
        const float npz = __fadd_rn(__fmul_rn(n[2], noise_pos), 0.0f);
        const float nvx = __fadd_rn(__fmul_rn(n[3], noise_vel), 0.0f);
        const float nvy = __fadd_rn(__fmul_rn(n[4], noise_vel), 0.0f);
        const float nvz = __fadd_rn(__fmul_rn(n[5], noise_vel), 0.0f);
        // pos += vel * dt + noise  (old velocity)
        px = __fadd_rn(px, __fadd_rn(__fmul_rn(vx, fp.dt), npx));
        py = __fadd_rn(py, __fadd_rn(__fmul_rn(vy, fp.dt), npy));
        pz = __fadd_rn(pz, __fadd_rn(__fmul_rn(vz, fp.dt), npz));
        vx = __fadd_rn(vx, nvx);
        vy = __fadd_rn(vy, nvy);
        vz = __fadd_rn(vz, nvz);
        w = __fmul_rn(w, p.p_S);
        const float lim = __fmul_rn(5.0f, p.init_max_vel);
        const float nlim = __fmul_rn(-5.0f, p.init_max_vel);
        vx = clampv(vx, nlim, lim);
        vy = clampv(vy, nlim, lim);
        vz = clampv(vz, nlim, lim);
        const int Gi = p.G, Gzi = p.Gz;
        const float G = (float)Gi, Gz = (float)Gzi;
        if ((px >= G || px < 0.0f) || (py >= G || py < 0.0f) || (pz >= Gz || pz < 0.0f)) w = 0.0f;
        const int ix = clampv(f2i_trunc(px), 0, Gi - 1);
        const int iy = clampv(f2i_trunc(py), 0, Gi - 1);
        const int iz = clampv(f2i_trunc(pz), 0, Gzi - 1);
        x[2 * (long)i] = make_float4(px, py, pz, vx);
        x[2 * (long)i + 1] = make_float4(vy, vz, w, __uint_as_float((uint32_t)a.assoc[i]));
        a.cell[i] = bt.off->cell[sc] + ix + Gi * iy + Gi * Gi * iz;
    }
}

void launch_predict(const Batch& bt, Particles a, float4* x, cudaStream_t st) {
    if (bt.P <= 0) return;
    ++g_launches;
    k_predict<<<div_up(bt.P, kBlock), kBlock, 0, st>>>(bt, a, x);
}

// Between the structure-of-arrays set and its 32-byte records (the layout k_predict writes).
__global__ void k_pack_records(int n, Particles a, float4* __restrict__ x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    x[2 * (long)i] = make_float4(a.px[i], a.py[i], a.pz[i], a.vx[i]);
    x[2 * (long)i + 1] = make_float4(a.vy[i], a.vz[i], a.w[i], __uint_as_float((uint32_t)a.assoc[i]));
}

__global__ void k_unpack_records(int n, const float4* __restrict__ x, Particles a) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 r0 = x[2 * (long)i], r1 = x[2 * (long)i + 1];
    a.px[i] = r0.x; a.py[i] = r0.y; a.pz[i] = r0.z; a.vx[i] = r0.w;
    a.vy[i] = r1.x; a.vz[i] = r1.y; a.w[i] = r1.z;
    a.assoc[i] = (uint8_t)__float_as_uint(r1.w);
}

void launch_pack_records(int n, Particles a, float4* x, cudaStream_t st) {
    if (n <= 0) return;
    ++g_launches;
    k_pack_records<<<div_up(n, kBlock), kBlock, 0, st>>>(n, a, x);
}

void launch_unpack_records(int n, const float4* x, Particles a, cudaStream_t st) {
    if (n <= 0) return;
    ++g_launches;
    k_unpack_records<<<div_up(n, kBlock), kBlock, 0, st>>>(n, x, a);
}

__global__ void k_shift_particles(int n, Particles a, int mx, int my, int mz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    a.px[i] = __fsub_rn(a.px[i], (float)mx);
    a.py[i] = __fsub_rn(a.py[i], (float)my);
    a.pz[i] = __fsub_rn(a.pz[i], (float)mz);
}

void launch_shift_particles(int n, Particles a, int mx, int my, int mz, cudaStream_t st) {
    if (n <= 0) return;
    ++g_launches;
    k_shift_particles<<<div_up(n, kBlock), kBlock, 0, st>>>(n, a, mx, my, mz);
}

// ---------------------------------------------------------------- gather + segmented sums
// After the sort: sorted slot i takes particle perm[i] (the payload permutation of
// thrust::sort_by_key, src/common/dom.cu:175-183). In the same pass the per-cell sums over the
// sorted ranges are formed -- the serial weight loop of gridCellPredictionUpdateKernel
// (src/k3dom/kernel/mass_update.cu:168-174) and the w*v sums behind statisticalMomentsKernel1/2
// (statistical_moments.cu:22-63) -- and the start/end ranges of particleToGridKernel
// (particle_to_grid.cu:23-39). The penalty of penalizeStaticParticlesKernel
// (resampling.cu:13-36) is recorded as the sign bit of the sorted weight and applied at
// resampling.
//
// Two levels. Each warp takes 128 sorted slots and finishes every cell whose particles lie in
// its range (FP64 segmented scan over 32-slot chunks). For a cell that crosses range boundaries
// it records the piece sums: the range's first piece (SegRec.lead) and its last piece
// (SegRec.trail). k_seg_fixup then adds, for each cell whose head lies in a range, that range's
// trail and the lead pieces of the following ranges up to the cell's end. Every sum is formed in
// a fixed order, so it is deterministic, and no warp walks a long cell alone.
constexpr int kSegItems = 4;                       // 32-wide chunks per warp range
constexpr int kSegRange = 32 * kSegItems;          // 128 sorted particles per warp
constexpr int kSegWarps = kBlock / 32;

long seg_rec_count(long P) { return P > 0 ? div_up(P, (long)kSegRange) : 1; }

struct SegVal {
    double w, x, y, z;
};

__device__ __forceinline__ SegVal shfl_up_seg(const SegVal& v, int d) {
    SegVal o;
    o.w = __shfl_up_sync(0xffffffffu, v.w, d);
    o.x = __shfl_up_sync(0xffffffffu, v.x, d);
    o.y = __shfl_up_sync(0xffffffffu, v.y, d);
    o.z = __shfl_up_sync(0xffffffffu, v.z, d);
    return o;
}

__device__ __forceinline__ void put_sums(CellWork cw, uint32_t key, double w, double x, double y, double z, int start,
                                         int end) {
    cw.sum_w[key] = (float)w;
    cw.sum_wvx[key] = (float)x;
    cw.sum_wvy[key] = (float)y;
    cw.sum_wvz[key] = (float)z;
    cw.start[key] = start;
    cw.end[key] = end;
}

// 4 CTAs per SM (64 registers): more particles' loads in flight than at the 74 registers the
// kernel takes unbounded (assignment 0.324 -> 0.311 ms on the config-1 frame)
__global__ void __launch_bounds__(kBlock, 4)
k_gather_segsum(Batch bt, const float4* __restrict__ x, Particles s, const uint32_t* __restrict__ keys,
                const uint32_t* __restrict__ perm, CellWork cw, SegRec* __restrict__ rec) {
    const int lane = threadIdx.x & 31;
    const long warp_global = (long)blockIdx.x * kSegWarps + (threadIdx.x >> 5);
    const long r0 = warp_global * kSegRange;
    const long P = bt.P;
    if (r0 >= P) return;
    const long r1 = min(r0 + (long)kSegRange, P);

    // carried state of the open segment (ends of the previous chunk); head -1: the segment
    // began before this range
    SegVal carry = {0.0, 0.0, 0.0, 0.0};
    long carry_head = -1;
    uint32_t prev_key = (r0 > 0) ? keys[r0 - 1] : 0xFFFFFFFFu;
    bool lead_open = true;  // the range's first piece has not ended yet
    if (lane == 0) {
        rec[warp_global].lead_end = -1;
        rec[warp_global].trail_head = -1;
    }
    __syncwarp();
    // the particles of one 32-slot chunk, loaded one chunk ahead of their stores (the next chunk's
    // loads are in flight while this one is stored and scanned)
    struct Chunk {
        uint32_t key, next_key;
        float px, py, pz, vx, vy, vz, w;
        uint8_t assoc;
    };
    auto load_chunk = [&](long c0) {
        Chunk c;
        const long pos = c0 + lane;
        const bool valid = pos < r1;
        c.key = valid ? keys[pos] : 0xFFFFFFFEu;
        c.next_key = (pos + 1 < P) ? keys[pos + 1] : 0xFFFFFFFDu;
        if (valid) {
            const long src = perm[pos];
            const float4 r0 = x[2 * src], r1 = x[2 * src + 1];  // one 32-byte sector
            c.px = r0.x; c.py = r0.y; c.pz = r0.z; c.vx = r0.w;
            c.vy = r1.x; c.vz = r1.y; c.w = r1.z;
            c.assoc = (uint8_t)__float_as_uint(r1.w);
        }
        return c;
    };
    Chunk nxt = load_chunk(r0);
#pragma unroll 1
    for (int it = 0; it < kSegItems; ++it) {
        const long c0 = r0 + 32L * it;
        if (c0 >= r1) break;
        const Chunk cur = nxt;
        if (c0 + 32 < r1) nxt = load_chunk(c0 + 32);
        const long pos = c0 + lane;
        const bool valid = pos < r1;
        const uint32_t key = cur.key;
        uint32_t kprev = __shfl_up_sync(0xffffffffu, key, 1);
        if (lane == 0) kprev = prev_key;
        prev_key = __shfl_sync(0xffffffffu, key, 31);
        const bool head = valid && (pos == 0 || key != kprev);
        const bool tail = valid && (key != cur.next_key);

        SegVal v = {0.0, 0.0, 0.0, 0.0};
        if (valid) {
            const float vx = cur.vx, vy = cur.vy, vz = cur.vz, w = cur.w;
            // sorted slots of a scene lie in its particle range (cells are scene-major)
            const float mv = bt.sc[scene_of(bt.off->part, bt.S, (int)pos)].p.min_vel;
            const float sp = __fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)), __fmul_rn(vz, vz));
            const bool slow = sp < __fmul_rn(mv, mv);
            s.px[pos] = cur.px;
            s.py[pos] = cur.py;
            s.pz[pos] = cur.pz;
            s.vx[pos] = vx;
            s.vy[pos] = vy;
            s.vz[pos] = vz;
            s.w[pos] = slow ? -w : w;  // sign bit = penalised at resampling
            s.assoc[pos] = cur.assoc;
            s.cell[pos] = (int)key;
            v.w = (double)w;
            v.x = (double)__fmul_rn(w, vx);
            v.y = (double)__fmul_rn(w, vy);
            v.z = (double)__fmul_rn(w, vz);
        }
        // segmented inclusive scan with head flags
        bool hf = head;
        long hpos = head ? pos : -1;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            SegVal o = shfl_up_seg(v, d);
            bool ohf = __shfl_up_sync(0xffffffffu, hf, d);
            long oh = __shfl_up_sync(0xffffffffu, hpos, d);
            if (lane >= d) {
                if (!hf) { v.w += o.w; v.x += o.x; v.y += o.y; v.z += o.z; }
                hf = hf || ohf;
                hpos = max(hpos, oh);
            }
        }
        if (!hf) {
            v.w += carry.w; v.x += carry.x; v.y += carry.y; v.z += carry.z;
            hpos = carry_head;
        }
        if (tail) {
            if (hpos >= 0) {
                put_sums(cw, key, v.w, v.x, v.y, v.z, (int)hpos, (int)pos);
            } else {
                // end of the range's first piece, whose cell began in an earlier range
                SegRec& r = rec[warp_global];
                r.lead[0] = v.w; r.lead[1] = v.x; r.lead[2] = v.y; r.lead[3] = v.z;
                r.lead_end = (int)pos;
            }
        }
        const int last = (int)min(31L, r1 - 1 - c0);  // last valid lane of the chunk
        carry.w = __shfl_sync(0xffffffffu, v.w, last);
        carry.x = __shfl_sync(0xffffffffu, v.x, last);
        carry.y = __shfl_sync(0xffffffffu, v.y, last);
        carry.z = __shfl_sync(0xffffffffu, v.z, last);
        carry_head = __shfl_sync(0xffffffffu, hpos, last);
        const bool last_tail = __shfl_sync(0xffffffffu, tail, last);
        if (__any_sync(0xffffffffu, tail && hpos < 0)) lead_open = false;
        if (c0 + 32 >= r1 && !last_tail && lane == last) {
            // the range's last piece continues into the next range
            SegRec& r = rec[warp_global];
            if (carry_head >= 0) {
                r.trail[0] = v.w; r.trail[1] = v.x; r.trail[2] = v.y; r.trail[3] = v.z;
                r.trail_head = (int)carry_head;
            } else if (lead_open) {
                // the whole range lies inside one cell that began earlier: all of it is lead
                r.lead[0] = v.w; r.lead[1] = v.x; r.lead[2] = v.y; r.lead[3] = v.z;
            }
        }
    }
}

// Cells that cross range boundaries: the range holding the head adds its trail and the
// following ranges' lead pieces in order until the piece that ends the cell.
__global__ void __launch_bounds__(kBlock)
k_seg_fixup(long nrec, const SegRec* __restrict__ rec, const uint32_t* __restrict__ keys, CellWork cw) {
    const long w = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= nrec) return;
    const int head = rec[w].trail_head;
    if (head < 0) return;
    double sw = rec[w].trail[0], sx = rec[w].trail[1], sy = rec[w].trail[2], sz = rec[w].trail[3];
    int end = -1;
    for (long v = w + 1; v < nrec; ++v) {
        sw += rec[v].lead[0];
        sx += rec[v].lead[1];
        sy += rec[v].lead[2];
        sz += rec[v].lead[3];
        if (rec[v].lead_end >= 0) {
            end = rec[v].lead_end;
            break;
        }
    }
    put_sums(cw, keys[head], sw, sx, sy, sz, head, end);
}

void launch_gather_segsum(const Batch& bt, const float4* x, Particles s, const uint32_t* sorted_keys,
                          const uint32_t* perm, CellWork cw, SegRec* rec, cudaStream_t st) {
    if (bt.P <= 0) return;
    const long warps = div_up((long)bt.P, (long)kSegRange);
    g_launches += 2;
    k_gather_segsum<<<div_up(warps, (long)kSegWarps), kBlock, 0, st>>>(bt, x, s, sorted_keys, perm, cw, rec);
    k_seg_fixup<<<div_up(warps, (long)kBlock), kBlock, 0, st>>>(warps, rec, sorted_keys, cw);
}

// ---------------------------------------------------------------- persistent reweight
// updatePersistentParticlesKernel3 (update_persistent_particles.cu:46-55) with p_A = 0:
// w = mu_UA * w. For DS-PHD/MIB the in-place normalisation of
// src/dsphdmib/kernel/mass_update.cu:37-44,64-68 (w /= occ_pred when the cell's weight
// sum exceeds 1) is applied first. The penalty flag (sign bit) is kept.
__global__ void __launch_bounds__(kBlock)
k_reweight(int P, int variant, Particles s, const uint32_t* __restrict__ keys, CellWork cw) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < P; i += gridDim.x * blockDim.x) {
    const uint32_t c = keys[i];
    const float wv = s.w[i];
    const bool flag = signbit(wv);
    float w = fabsf(wv);
    if (variant == 1) {
        const float d = cw.divisor[c];
        if (d > 0.0f) w = __fdiv_rn(w, d);
    }
    // p_A * mu_A * post_w + (1 - p_A) * mu_UA * w with p_A = 0, likelihood = 1
    const float f = cw.factor[c];
    w = __fadd_rn(0.0f, __fmul_rn(f, w));
    s.w[i] = flag ? -w : w;
  }
}

void launch_reweight(const Batch& bt, Particles s, const uint32_t* sorted_keys, CellWork cw,
                     cudaStream_t st) {
    if (bt.P <= 0) return;
    ++g_launches;
    k_reweight<<<grid_for(bt.P), kBlock, 0, st>>>(bt.P, bt.variant, s, sorted_keys, cw);
}

// ---------------------------------------------------------------- slot ownership
// Slot ranges of init_new_particles.cu:14-27: cell j owns slots
// [int(acc[j-1]*k), int(acc[j]*k) - 1] with k = v / acc[C-1] (normalize_particle_orders,
// :44-52). bound(j) = int(acc[j] * k) is monotone in j.
struct SlotMap {
    const float* cum;
    int C;
    float k;
    __device__ __forceinline__ int bound(int j) const { return f2i_trunc(__fmul_rn(cum[j], k)); }
    // first j with bound(j) > s, or C when none
    __device__ __forceinline__ int owner(int s) const {
        int lo = 0, hi = C;
        while (lo < hi) {
            int mid = (lo + hi) >> 1;
            if (bound(mid) > s) hi = mid; else lo = mid + 1;
        }
        return lo;
    }
    __device__ __forceinline__ int start(int j) const { return j == 0 ? 0 : bound(j - 1); }
    __device__ __forceinline__ int count(int j) const {
        int st = start(j), en = bound(j) - 1;
        return st <= en ? en - st + 1 : 0;
    }
};

__device__ __forceinline__ SlotMap make_slotmap(const float* cum, int C, int v) {
    SlotMap m;
    m.cum = cum;
    m.C = C;
    const float mx = cum[C - 1];
    m.k = __fdiv_rn((float)v, mx);  // v_B / max
    return m;
}

// Uniform velocity in [-vmax, vmax) with the minimum-speed rescale
// (init_new_particles.cu:77-87, 147-167).
__device__ __forceinline__ void birth_velocity(float u0, float u1, float u2, float vmax, float min_vel,
                                               float* vx, float* vy, float* vz) {
    const float lo = -vmax, hi = vmax;
    const float span = __fsub_rn(hi, lo);
    float x = __fadd_rn(lo, __fmul_rn(span, __fsub_rn(1.0f, u0)));
    float y = __fadd_rn(lo, __fmul_rn(span, __fsub_rn(1.0f, u1)));
    float z = __fadd_rn(lo, __fmul_rn(span, __fsub_rn(1.0f, u2)));
    const float vsq = __fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z));
    if (vsq < __fmul_rn(min_vel, min_vel) && vsq != 0.0f) {
        const float rate = __fdiv_rn(min_vel, __fsqrt_rn(vsq));
        x = __fmul_rn(x, rate);
        y = __fmul_rn(y, rate);
        z = __fmul_rn(z, rate);
    }
    *vx = x; *vy = y; *vz = z;
}

__device__ __forceinline__ void cell_centre_idx(int c, int G, float* x, float* y, float* z) {
    int ix, iy, iz;
    cell_xyz(c, G, &ix, &iy, &iz);
    *x = __fadd_rn((float)ix, 0.5f);
    *y = __fadd_rn((float)iy, 0.5f);
    *z = __fadd_rn((float)iz, 0.5f);
}

// ---------------------------------------------------------------- births
// initNewParticlesKernel1/2 (init_new_particles.cu:106-183). One thread per birth slot
// finds its cell by binary search instead of each cell looping over its slots. Slots
// beyond the last cell's range keep the previous frame's cell and association, exactly as
// the reference leaves them unwritten. The penalty of penalizeStaticParticlesKernel
// (resampling.cu:35-42) is recorded in the sign bit of the weight.
__global__ void __launch_bounds__(kBlock)
k_births(Batch bt, const float* __restrict__ born, const float* __restrict__ cum, Particles b) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < bt.B; g += gridDim.x * blockDim.x) {
        const int sc = scene_of(bt.off->birth, bt.S, g);
        const DevParams& p = bt.sc[sc].p;
        const FrameParams& fp = bt.fp[sc];
        const int s = g - bt.off->birth[sc];  // slot within the scene
        const int coff = bt.off->cell[sc];
        const int C = p.C;
        const float p_A = p.p_A;
        const SlotMap m = make_slotmap(cum + coff, C, p.B);
        int j = m.owner(s);
        bool assoc;
        int n, st;
        if (j < C) {
            st = m.start(j);
            n = m.bound(j) - 1 - st + 1;
            const int nu_A0 = (int)roundf(__fmul_rn((float)n, p_A));
            assoc = s < st + nu_A0;
            b.cell[g] = coff + j;
            b.assoc[g] = assoc ? 1 : 0;
        } else {
            j = clampv(b.cell[g] - coff, 0, C - 1);
            assoc = b.assoc[g] != 0;
            n = m.count(j);
        }
        const int nu_A = (int)roundf(__fmul_rn((float)n, p_A));
        const int nu_UA = n - nu_A;
        const float bm = born[coff + j];
        float w;
        if (assoc) {
            w = nu_A > 0 ? __fdiv_rn(__fmul_rn(p_A, bm), (float)nu_A) : 0.0f;
        } else {
            w = nu_UA > 0 ? (float)((1.0 - (double)p_A) * (double)bm / (double)nu_UA) : 0.0f;
        }
        float x, y, z, vx, vy, vz;
        cell_centre_idx(j, p.G, &x, &y, &z);
        const U4 r = block(fp.seed, fp.frame, kBirthVel, (uint64_t)s, 0);
        const float min_vel = p.min_vel;
        birth_velocity(u01(r.x), u01(r.y), u01(r.z), p.init_max_vel, min_vel, &vx, &vy, &vz);
        const float sp = __fadd_rn(__fadd_rn(__fmul_rn(vx, vx), __fmul_rn(vy, vy)), __fmul_rn(vz, vz));
        const bool slow = sp < __fmul_rn(min_vel, min_vel);
        b.px[g] = x; b.py[g] = y; b.pz[g] = z;
        b.vx[g] = vx; b.vy[g] = vy; b.vz[g] = vz;
        b.w[g] = slow ? -w : w;
    }
}

void launch_births(const Batch& bt, const float* born, const float* born_cum, Particles b, cudaStream_t st) {
    if (bt.B <= 0) return;
    ++g_launches;
    k_births<<<grid_for(bt.B), kBlock, 0, st>>>(bt, born, born_cum, b);
}

// ---------------------------------------------------------------- first frame
// initParticlesKernel1/2 (init_new_particles.cu:54-104) driven by the born-mass prefix
// normalised to P (src/k3dom/dom.cu:60-76, src/dsphdmib/dom.cu:65-81).
__global__ void __launch_bounds__(kBlock)
k_init_particles(Batch bt, const float* __restrict__ cum, Particles a) {
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < bt.P; g += gridDim.x * blockDim.x) {
        const int sc = scene_of(bt.off->part, bt.S, g);
        const DevParams& p = bt.sc[sc].p;
        const FrameParams& fp = bt.fp[sc];
        const int s = g - bt.off->part[sc];
        const int coff = bt.off->cell[sc];
        const int C = p.C, P = p.P;
        const SlotMap m = make_slotmap(cum + coff, C, P);
        int j = m.owner(s);
        if (j < C) {
            a.cell[g] = coff + j;
        } else {
            j = clampv(a.cell[g] - coff, 0, C - 1);
        }
        float x, y, z, vx, vy, vz;
        cell_centre_idx(j, p.G, &x, &y, &z);
        const U4 r = block(fp.seed, fp.frame, kInitVel, (uint64_t)s, 0);
        birth_velocity(u01(r.x), u01(r.y), u01(r.z), p.init_max_vel, p.min_vel, &vx, &vy, &vz);
        a.px[g] = x; a.py[g] = y; a.pz[g] = z;
        a.vx[g] = vx; a.vy[g] = vy; a.vz[g] = vz;
        a.w[g] = __fdiv_rn(1.0f, (float)P);
    }
}

void launch_init_particles(const Batch& bt, const float* born_cum, Particles a, cudaStream_t st) {
    if (bt.P <= 0) return;
    ++g_launches;
    k_init_particles<<<grid_for(bt.P), kBlock, 0, st>>>(bt, born_cum, a);
}

// ---------------------------------------------------------------- resampling
// Resampling draws as 24-bit keys of 1 - u: sorting the keys ascending orders the draws
// u * joint_max ascending for any joint_max >= 0, so the draws can be sorted before the
// weights exist (resamplingGenerateRandomNumbersKernel + thrust::sort, resampling.cu:38-53,
// src/common/dom.cu:277-285). The scene index sits above the 24 key bits, so one sort orders
// every scene's draws within the scene's own particle range.
__global__ void k_draw_keys(Batch bt, uint32_t* keys) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < bt.P; i += gridDim.x * blockDim.x) {
        const int sc = scene_of(bt.off->part, bt.S, i);
        const FrameParams& fp = bt.fp[sc];
        const int local = i - bt.off->part[sc];
        keys[i] = ((uint32_t)sc << 24) | one_minus_u01_key(resample_word(fp.seed, fp.frame, (uint64_t)local));
    }
}

int draw_key_bits(int S) {
    int b = 0;
    while ((1 << b) < S) ++b;
    return 24 + b;
}

void launch_draw_keys(const Batch& bt, uint32_t* keys, cudaStream_t st) {
    if (bt.P <= 0) return;
    ++g_launches;
    k_draw_keys<<<grid_for(bt.P), kBlock, 0, st>>>(bt, keys);
}

constexpr int kResThreads = 256;

// calc_resampled_indices + resamplingKernel (resampling.cu:55-89): ancestor =
// lower_bound(acc, u) where acc's last element is replaced by the largest draw when they
// differ; the resampled particle is gathered from the sorted persistent set or the birth
// set with weight joint_max / P. Ancestors are scene-local indices into [persistent, births).
struct ResScene {
    const float* cum;
    int n, P;
    float jmax, rmax;
    const uint32_t* dk;  // the scene's sorted draw keys
    __device__ __forceinline__ float acc(int j) const { return j == n - 1 ? rmax : cum[j]; }
    __device__ __forceinline__ int lower(float u, int lo, int hi) const {  // first j in [lo, hi) with acc[j] >= u
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (acc(mid) < u) lo = mid + 1; else hi = mid;
        }
        return lo;
    }
    __device__ __forceinline__ float draw(int k) const {  // k local
        const float om = (float)(dk[k] & 0xFFFFFFu) * 5.9604644775390625e-08f;
        return __fadd_rn(0.0f, __fmul_rn(jmax, om));
    }
};

__device__ __forceinline__ ResScene res_scene(const Batch& bt, const float* joint_cum, const uint32_t* dkeys, int sc) {
    ResScene r;
    const DevParams& p = bt.sc[sc].p;
    r.P = p.P;
    r.n = p.P + p.B;
    r.cum = joint_cum + bt.off->joint[sc];
    r.dk = dkeys + bt.off->part[sc];
    r.jmax = r.cum[r.n - 1];
    const float om_max = (float)(r.dk[r.P - 1] & 0xFFFFFFu) * 5.9604644775390625e-08f;
    r.rmax = __fadd_rn(0.0f, __fmul_rn(r.jmax, om_max));
    return r;
}

constexpr int kResPerThread = 4;
constexpr int kResBlock = kResThreads * kResPerThread;  // draws per resampling block

long res_bracket_count(long P) { return P > 0 ? div_up(P, (long)kResBlock) : 1; }

// The block's draws are sorted, so its ancestors lie in [lower(first draw), lower(last draw)]:
// one warp per end of each block's bracket (all blocks in parallel). joint_cum is an exactly
// rounded prefix of non-negative weights, hence non-decreasing, and every draw is at most the
// replaced last entry, so "acc(j) >= u" is false then true along the whole range and a 33-way
// search (32 probes per step, about 4 dependent loads for a million entries instead of ~20)
// returns the same index as the binary search. A block whose draws span two scenes gets
// (-1, -1) and searches each draw in full.
__global__ void k_res_brackets(Batch bt, const float* __restrict__ joint_cum, const uint32_t* __restrict__ dkeys,
                               int nblocks, int* __restrict__ br) {
    const int w = (int)(((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    const int blk = w >> 1, end = w & 1;
    if (blk >= nblocks) return;  // whole warps leave together
    const int k0 = blk * kResBlock;
    const int k1 = min(k0 + kResBlock, bt.P) - 1;
    const int sc = scene_of(bt.off->part, bt.S, k0);
    if (scene_of(bt.off->part, bt.S, k1) != sc) {
        if (lane == 0) br[w] = -1;
        return;
    }
    const ResScene r = res_scene(bt, joint_cum, dkeys, sc);
    const float u = r.draw((end ? k1 : k0) - bt.off->part[sc]);
    int lo = 0, hi = r.n;  // answer in [lo, hi]; hi when no entry of [lo, hi) reaches u
    while (hi - lo > 32) {
        const long span = hi - lo;
        const int pos = lo + (int)(((long)(lane + 1) * span) / 33);  // strictly increasing, in [lo, hi)
        const unsigned m = __ballot_sync(0xFFFFFFFFu, r.acc(pos) >= u);
        const int f = m ? __ffs(m) - 1 : 32;
        const int prev = __shfl_sync(0xFFFFFFFFu, pos, f > 0 ? f - 1 : 0);
        const int at = __shfl_sync(0xFFFFFFFFu, pos, f < 32 ? f : 0);
        if (f < 32) hi = at;
        if (f > 0) lo = prev + 1;
    }
    const int pos = lo + lane;
    const unsigned m = __ballot_sync(0xFFFFFFFFu, pos < hi && r.acc(pos) >= u);
    if (lane == 0) br[w] = m ? lo + __ffs(m) - 1 : hi;
}

constexpr int kResStage = 4096;  // bracket entries staged in shared memory

// One resampled particle: the ancestor's state, gathered before any store so that the loads of
// a thread's draws are all in flight together.
struct ResPart {
    float px, py, pz, vx, vy, vz;
    int cell;
    uint8_t assoc;
};

__device__ __forceinline__ int res_clamp(const ResScene& r, int a) { return a > r.n - 1 ? r.n - 1 : a; }

__device__ __forceinline__ ResPart res_load(const Batch& bt, const ResScene& r, int sc, int a, const Particles& s,
                                            const Particles& b) {
    ResPart v;
    const bool pers = a < r.P;
    const int q = pers ? bt.off->part[sc] + a : bt.off->birth[sc] + a - r.P;
    const Particles& src = pers ? s : b;
    v.px = src.px[q]; v.py = src.py[q]; v.pz = src.pz[q];
    v.vx = src.vx[q]; v.vy = src.vy[q]; v.vz = src.vz[q];
    v.cell = src.cell[q];
    v.assoc = src.assoc[q];
    return v;
}

__device__ __forceinline__ void res_store(const ResScene& r, int k, int a, const ResPart& v, Particles& out,
                                          int* __restrict__ anc_out) {
    out.px[k] = v.px; out.py[k] = v.py; out.pz[k] = v.pz;
    out.vx[k] = v.vx; out.vy[k] = v.vy; out.vz[k] = v.vz;
    out.cell[k] = v.cell;
    out.assoc[k] = v.assoc;
    out.w[k] = __fdiv_rn(r.jmax, (float)r.P);
    anc_out[k] = a;
}

// 5 CTAs per SM (48 registers, no spills): the gathers through the ancestor index wait on memory
// latency, so more resident warps help.
__global__ void __launch_bounds__(kResThreads, 5)
k_resample(Batch bt, const float* __restrict__ joint_cum, const uint32_t* __restrict__ dkeys, const int2* br,
           Particles s, Particles b, Particles out, int* __restrict__ anc_out, float* __restrict__ joint_max_out) {
    __shared__ float s_acc[kResStage];
    const int k0 = blockIdx.x * kResBlock;
    const int2 bk = br[blockIdx.x];
    if (bk.x >= 0) {
        const int sc = scene_of(bt.off->part, bt.S, k0);
        const ResScene r = res_scene(bt, joint_cum, dkeys, sc);
        const int base = bt.off->part[sc];
        // search the bracket [lo, hi]; staged in shared memory when it fits (block-uniform)
        const int lo = bk.x, hi = min(bk.y + 1, r.n), len = hi - lo;
        const bool staged = len <= kResStage;
        if (staged) {
            for (int i = threadIdx.x; i < len; i += kResThreads) s_acc[i] = r.acc(lo + i);
            __syncthreads();
        }
        int a[kResPerThread];
#pragma unroll
        for (int it = 0; it < kResPerThread; ++it) {
            const int k = k0 + it * kResThreads + threadIdx.x;
            a[it] = 0;
            if (k >= bt.P) continue;
            const float u = r.draw(k - base);
            if (staged) {
                int l = 0, h = len;  // first j in [0, len) with s_acc[j] >= u
                while (l < h) {
                    const int mid = (l + h) >> 1;
                    if (s_acc[mid] < u) l = mid + 1; else h = mid;
                }
                a[it] = res_clamp(r, lo + l);
            } else {
                a[it] = res_clamp(r, r.lower(u, lo, hi));
            }
        }
        ResPart v[kResPerThread];
#pragma unroll
        for (int it = 0; it < kResPerThread; ++it)
            if (k0 + it * kResThreads + (int)threadIdx.x < bt.P) v[it] = res_load(bt, r, sc, a[it], s, b);
#pragma unroll
        for (int it = 0; it < kResPerThread; ++it) {
            const int k = k0 + it * kResThreads + threadIdx.x;
            if (k >= bt.P) continue;
            res_store(r, k, a[it], v[it], out, anc_out);
            if (k == base && joint_max_out) joint_max_out[sc] = r.jmax;
        }
    } else {
        for (int it = 0; it < kResPerThread; ++it) {
            const int k = k0 + it * kResThreads + threadIdx.x;
            if (k >= bt.P) break;
            const int sc = scene_of(bt.off->part, bt.S, k);
            const ResScene r = res_scene(bt, joint_cum, dkeys, sc);
            const int kl = k - bt.off->part[sc];
            const int a = res_clamp(r, r.lower(r.draw(kl), 0, r.n));
            res_store(r, k, a, res_load(bt, r, sc, a, s, b), out, anc_out);
            if (kl == 0 && joint_max_out) joint_max_out[sc] = r.jmax;
        }
    }
}

void launch_resample(const Batch& bt, const float* joint_cum, const uint32_t* sorted_draws, Particles s,
                     Particles b, Particles out, int* ancestors, float* joint_max_out, int2* brackets,
                     cudaStream_t st) {
    if (bt.P <= 0) return;
    const int nblk = div_up(bt.P, kResBlock);
    g_launches += 2;
    k_res_brackets<<<div_up(nblk * 64, 256), 256, 0, st>>>(bt, joint_cum, sorted_draws, nblk,
                                                           reinterpret_cast<int*>(brackets));
    k_resample<<<nblk, kResThreads, 0, st>>>(bt, joint_cum, sorted_draws, brackets, s, b, out, ancestors,
                                             joint_max_out);
}

// ---------------------------------------------------------------- debug draws
__global__ void k_debug_draws(uint64_t seed, int frame, int stage, long first, long count, float* dst) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const uint64_t item = (uint64_t)(first + t);
    if (stage == kPredict) {
        float n[6];
        predict_normals(seed, (uint32_t)frame, item, n);
        for (int k = 0; k < 6; ++k) dst[t * 6 + k] = n[k];
    } else if (stage == kInitVel || stage == kBirthVel) {
        const U4 r = block(seed, (uint32_t)frame, (uint32_t)stage, item, 0);
        dst[t * 3 + 0] = u01(r.x);
        dst[t * 3 + 1] = u01(r.y);
        dst[t * 3 + 2] = u01(r.z);
    } else {
        dst[t] = u01(resample_word(seed, (uint32_t)frame, item));
    }
}

void launch_debug_draws(uint64_t seed, int frame, int stage, long first, long count, float* dst,
                        cudaStream_t st) {
    if (count <= 0) return;
    ++g_launches;
    k_debug_draws<<<div_up(count, kBlock), kBlock, 0, st>>>(seed, frame, stage, first, count, dst);
}

}  // namespace k3dom
