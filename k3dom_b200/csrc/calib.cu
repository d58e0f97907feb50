// calib.cu -- the differentiable kernel-inference update: a calibration loss over held-out rays
// and its hand-written adjoint with respect to the kernel length-scale, the kernel amplitude,
// the free-space decay and the prior masses.
//
// Forward, per cell c (the K3DOM cell update of src/k3dom/kernel/mass_update.cu:79-183, in FP64):
//   frame 0: masses start at the priors (free = theta_free, static = dynamic = theta_occ / 2), are
//            predicted with dt = 0 and no particles, and updated with the BGKI evidence
//            E = sigma * sum f(d / ls) of the frame's scan (occupied and free parts);
//   frame k: predicted with gamma^dt_k and the frame's particle weight sum (given, not
//            differentiated: sort and resampling are not differentiable), then updated;
//   p(c) = (static + dynamic) / (free + static + dynamic) after the last frame.
// Loss = mean over held-out label instances of the binary cross-entropy of p(c) (p clamped to
// [1e-7, 1 - 1e-7]); labels come from 3-D DDA along each held-out ray: 1 for the voxel holding
// the hit, 0 for the voxels traversed before it.
//
// The free-space decay of the calibration is the reference's gamma (the only decay on free mass,
// pred_total = (free + dynamic) gamma^dt, mass_update.cu:166). The occupied prior is split
// evenly between the static and dynamic prior masses.
//
// Gradient: the evidence enters only through per-cell sums F = sum f(x) and H = sum -x f'(x)
// (x = d / ls), formed by one BGKI pass per frame (k_bgki_sums, exact fixed point, no per-pair
// storage): dE/dsigma = F, dE/dls = sigma H / ls. The backward recomputes each cell's mass
// recursion and runs it in reverse (frame_adjoint), then reduces sum_c dL/dE * dE/dtheta over the
// cells; nothing per point and nothing per frame intermediate is kept between the passes.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/k3dom_b200.h"
#include "common.cuh"
#include "internal.h"

using namespace k3dom;

namespace {

constexpr int kMaxCalibFrames = 16;
constexpr double kPClamp = 1e-7;

// ---------------------------------------------------------------- per-cell mass recursion
// k2 = 2 / mass_scale throughout.
// credit(x) = 1 - 2 / (1 + e), e = exp(2x / mass_scale)
__device__ inline double credit(double x, double k2) { return 1.0 - 2.0 / (1.0 + exp(x * k2)); }
// d credit / dx = (4 / ms) e / (1 + e)^2, written with t = exp(-|2x / ms|) (the same value,
// e / (1 + e)^2 = t / (1 + t)^2) so that it cannot overflow to inf / inf.
__device__ inline double credit_d(double x, double k2) {
    const double t = exp(-fabs(x * k2));
    const double u = 1.0 + t;
    return (2.0 * k2) * t / (u * u);
}

struct FrameIn {
    double mf, ms, md;  // masses entering the frame (before prediction)
    double g;           // gamma^dt
    double dyn;         // particle weight sum of the cell (0 without particles)
    double Eo, Ef;      // evidence
};

// The evidence-driven transfers of the update (mass_update.cu:95-118), shared by the forward and
// the adjoint's recomputation: with Z = Sd Sp, X = sqrt(Z), cr = credit(X) and w = cr / Z,
// lDF = w (Ef - Eo)+ d1, lSFD = w (Ef - Eo)+ (s1 + d1 - f1)+, lFD = w (Eo - Ef)+ (f1 - s1 - d1)+
// (the reference's bf d1 / Sp etc. with bf = cr (Ef - Eo)+ / Sd).
struct Transfers {
    double iZ, X, cr, w, lDF, lSFD, lFD;
};

__device__ inline Transfers transfers(double Eo, double Ef, double f1, double s1, double d1, double Sd,
                                      double Sp, double k2) {
    Transfers t = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (Sp > 0.0) {
        const double Z = Sd * Sp;
        t.iZ = 1.0 / Z;
        t.X = sqrt(Z);
        t.cr = credit(t.X, k2);
        t.w = t.cr * t.iZ;
        const double pf = fmax(0.0, Ef - Eo), po = fmax(0.0, Eo - Ef);
        t.lDF = t.w * pf * d1;
        t.lSFD = t.w * pf * fmax(0.0, s1 + d1 - f1);
        t.lFD = t.w * po * fmax(0.0, f1 - s1 - d1);
    }
    return t;
}

// The frame's prediction and update (mass_update.cu:79-139), FP64.
__device__ inline void frame_forward(const FrameIn& in, double k2, double* f3, double* s3, double* d3) {
    const double P = (in.mf + in.md) * in.g;
    const double s1 = in.ms * in.g;
    const double d1 = fmin(in.dyn, fmax(0.0, P - s1));
    const double f1 = P - d1;
    if (!(in.Ef > 0.0 || in.Eo > 0.0)) {
        *f3 = f1; *s3 = s1; *d3 = d1;
        return;
    }
    const Transfers t = transfers(in.Eo, in.Ef, f1, s1, d1, in.Ef + in.Eo, f1 + s1 + d1, k2);
    const double f2 = f1 + t.lSFD / 2.0 * s1 + t.lDF * d1 - t.lFD * f1;
    const double s2 = s1 - t.lSFD * s1;
    const double d2 = d1 + t.lFD * f1 + t.lSFD / 2.0 * s1 - t.lDF * d1;
    const double y = s2 + d2;
    const double cr2 = credit(y, k2);
    // ratio 1 / (1 + d2 / s2) = s2 / (s2 + d2)
    const double r = (s2 <= 0.0 || d2 < 0.0) ? 0.0 : s2 / y;
    const double beta = (1.0 - cr2) + cr2 * r;
    *s3 = s2 + beta * in.Eo;
    *d3 = d2 + (1.0 - beta) * in.Eo;
    *f3 = f2 + in.Ef;
}

struct FrameBar {
    double mf, ms, md, g, Eo, Ef;
};

// Reverse mode of frame_forward: adjoints of the outputs (F3, S3, D3) -> adjoints of the inputs.
// Piecewise branches (min, max, the update condition, the ratio's guard) take the derivative of
// the branch the forward took.
__device__ inline FrameBar frame_adjoint(const FrameIn& in, double k2, double F3, double S3, double D3) {
    FrameBar b = {0, 0, 0, 0, 0, 0};
    // forward recomputation
    const double P = (in.mf + in.md) * in.g;
    const double s1 = in.ms * in.g;
    const double t = P - s1;
    const double u = fmax(0.0, t);
    const bool d_is_dyn = in.dyn < u;
    const double d1 = d_is_dyn ? in.dyn : u;
    const double f1 = P - d1;
    double f1b = 0.0, s1b = 0.0, d1b = 0.0;
    if (!(in.Ef > 0.0 || in.Eo > 0.0)) {
        f1b = F3; s1b = S3; d1b = D3;
    } else {
        const double Sd = in.Ef + in.Eo;
        const double Sp = f1 + s1 + d1;
        const double pf = fmax(0.0, in.Ef - in.Eo), po = fmax(0.0, in.Eo - in.Ef);
        const double q1 = fmax(0.0, s1 + d1 - f1), q2 = fmax(0.0, f1 - s1 - d1);
        const Transfers tr = transfers(in.Eo, in.Ef, f1, s1, d1, Sd, Sp, k2);
        const double lDF = tr.lDF, lSFD = tr.lSFD, lFD = tr.lFD;
        const double s2 = s1 - lSFD * s1;
        const double d2 = d1 + lFD * f1 + lSFD / 2.0 * s1 - lDF * d1;
        const double y = s2 + d2;
        const double cr2 = credit(y, k2);
        const bool r_on = !(s2 <= 0.0 || d2 < 0.0);
        const double iy = r_on ? 1.0 / y : 0.0;
        const double r = s2 * iy;
        const double beta = (1.0 - cr2) + cr2 * r;
        // reverse
        double f2b = F3, s2b = S3, d2b = D3;
        b.Ef += F3;
        const double betab = in.Eo * (S3 - D3);
        b.Eo += S3 * beta + D3 * (1.0 - beta);
        const double cr2b = betab * (r - 1.0);
        const double rb = betab * cr2;
        const double yb = cr2b * credit_d(y, k2);
        s2b += yb;
        d2b += yb;
        if (r_on) {
            // r = s2 / (s2 + d2): dr/ds2 = d2 / y^2, dr/dd2 = -s2 / y^2
            const double riy2 = rb * iy * iy;
            s2b += riy2 * d2;
            d2b -= riy2 * s2;
        }
        double lSFDb = 0.0, lDFb = 0.0, lFDb = 0.0;
        // f2 = f1 + lSFD/2 s1 + lDF d1 - lFD f1
        f1b += f2b * (1.0 - lFD);
        s1b += f2b * lSFD / 2.0;
        d1b += f2b * lDF;
        lSFDb += f2b * s1 / 2.0;
        lDFb += f2b * d1;
        lFDb += -f2b * f1;
        // s2 = s1 - lSFD s1
        s1b += s2b * (1.0 - lSFD);
        lSFDb += -s2b * s1;
        // d2 = d1 + lFD f1 + lSFD/2 s1 - lDF d1
        d1b += d2b * (1.0 - lDF);
        f1b += d2b * lFD;
        s1b += d2b * lSFD / 2.0;
        lFDb += d2b * f1;
        lSFDb += d2b * s1 / 2.0;
        lDFb += -d2b * d1;
        if (Sp > 0.0) {
            // lDF = w pf d1, lSFD = w pf q1, lFD = w po q2, w = cr / (Sd Sp), cr = credit(sqrt(Sd Sp))
            const double w = tr.w;
            const double pfb = w * (lDFb * d1 + lSFDb * q1);
            const double pob = w * lFDb * q2;
            d1b += lDFb * w * pf;
            const double q1b = lSFDb * w * pf;
            const double q2b = lFDb * w * po;
            const double wb = lDFb * pf * d1 + lSFDb * pf * q1 + lFDb * po * q2;
            // w = cr / Z, Z = Sd Sp: crb = wb / Z, Zb = -wb w / Z; X = sqrt(Z): Zb += Xb / (2 X)
            const double crb = wb * tr.iZ;
            double Zb = -wb * w * tr.iZ;
            const double Xb = crb * credit_d(tr.X, k2);
            if (tr.X > 0.0) Zb += Xb / (2.0 * tr.X);
            if (s1 + d1 - f1 > 0.0) { s1b += q1b; d1b += q1b; f1b -= q1b; }
            if (f1 - s1 - d1 > 0.0) { f1b += q2b; s1b -= q2b; d1b -= q2b; }
            if (in.Ef - in.Eo > 0.0) { b.Ef += pfb; b.Eo -= pfb; }
            if (in.Eo - in.Ef > 0.0) { b.Eo += pob; b.Ef -= pob; }
            const double Sdb = Zb * Sp, Spb = Zb * Sd;
            f1b += Spb; s1b += Spb; d1b += Spb;
            b.Ef += Sdb; b.Eo += Sdb;
        }
    }
    // prediction reverse: f1 = P - d1; d1 = min(dyn, u); u = max(0, t); t = P - s1
    double Pb = f1b;
    d1b -= f1b;
    if (!d_is_dyn) {
        const double ub = d1b;
        if (t > 0.0) {
            Pb += ub;
            s1b -= ub;
        }
    }
    b.ms += s1b * in.g;
    b.g += s1b * in.ms + Pb * (in.mf + in.md);
    b.mf += Pb * in.g;
    b.md += Pb * in.g;
    return b;
}

// Frame k's sums of cell c as (F occ, F free, H occ, H free), FP64: the exact 64-bit unit sums
// times 2^-kCalibShift (a power of two, so the conversion is exact up to 2^53 units).
__device__ __forceinline__ double4 frame_sums(const long long* __restrict__ acc, long C, int k, long c) {
    const longlong2* p = reinterpret_cast<const longlong2*>(acc + (((long)k * C + c) << 2));
    const longlong2 a = p[0], b = p[1];
    const double u = 1.0 / (double)(1ull << kCalibShift);
    return make_double4((double)a.x * u, (double)a.y * u, (double)b.x * u, (double)b.y * u);
}

struct CalibCellArgs {
    int C, F;
    double ls, sigma, gamma, prior_occ, prior_free;
    double k2;  // 2 / mass_scale
    double inv_n;  // 1 / number of label instances
    double g[kMaxCalibFrames];   // gamma^dt of each frame (1 for the first)
    double gd[kMaxCalibFrames];  // d gamma^dt / d gamma (0 for the first frame and for dt = 0)
    const float* dyn[kMaxCalibFrames];  // per frame: particle weight sums (nullptr = none)
    const long long* acc;               // F x C x 4 units of 2^-kCalibShift: f occ, f free, -x f' occ, -x f' free
    const uint32_t* n0;
    const uint32_t* n1;
    float* occ_out;  // optional
    double* red;     // [0] loss, [1..5] gradient of (ls, sigma, gamma, prior_occ, prior_free)
    int want_grad;
};

__device__ inline double block_sum(double v, double* sm) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sm[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r += sm[i];
    return r;  // valid in thread 0
}

// NF: compile-time bound on the frame count. Up to 4 frames the loops unroll and the per-frame
// inputs stay in registers; the 16-frame form keeps them in local memory.
template <int NF>
__global__ void __launch_bounds__(256) k_calib_cells(CalibCellArgs a) {
    __shared__ double sm[8];
    double loss = 0.0, g_ls = 0.0, g_sig = 0.0, g_gam = 0.0, g_po = 0.0, g_pf = 0.0;
    const long C = a.C;
    for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < C; c += (long)gridDim.x * blockDim.x) {
        const uint32_t n0 = a.n0[c], n1 = a.n1[c];
        const bool labelled = (n0 | n1) != 0;
        if (!labelled && !a.occ_out) continue;
        FrameIn in[NF];
        double mf = a.prior_free, ms = a.prior_occ / 2.0, md = a.prior_occ / 2.0;
#pragma unroll(NF <= 4 ? NF : 1)
        for (int k = 0; k < NF; ++k) {
            if (k < a.F) {
                const double4 s = frame_sums(a.acc, C, k, c);
                FrameIn& x = in[k];
                x.mf = mf; x.ms = ms; x.md = md;
                x.g = a.g[k];
                x.dyn = (k == 0 || !a.dyn[k]) ? 0.0 : (double)a.dyn[k][c];
                x.Eo = a.sigma * s.x;
                x.Ef = a.sigma * s.y;
                frame_forward(x, a.k2, &mf, &ms, &md);
            }
        }
        const double T = mf + ms + md;
        const double iT = T > 0.0 ? 1.0 / T : 0.0;
        const double p = T > 0.0 ? (ms + md) * iT : 0.5;
        if (a.occ_out) a.occ_out[c] = (float)p;
        if (!labelled) continue;
        const double pc = fmin(fmax(p, kPClamp), 1.0 - kPClamp);
        loss += -(double)n1 * log(pc) - (double)n0 * log(1.0 - pc);
        if (!a.want_grad) continue;
        double pb = (p > kPClamp && p < 1.0 - kPClamp) ? (-(double)n1 / pc + (double)n0 / (1.0 - pc)) : 0.0;
        pb *= a.inv_n;
        double Fb = 0.0, Sb = 0.0, Db = 0.0;
        if (T > 0.0) {
            const double pbT2 = pb * iT * iT;
            Fb = -pbT2 * (ms + md);
            Sb = pbT2 * mf;
            Db = Sb;
        }
#pragma unroll(NF <= 4 ? NF : 1)
        for (int k = NF - 1; k >= 0; --k) {
            if (k < a.F) {
                const FrameBar b = frame_adjoint(in[k], a.k2, Fb, Sb, Db);
                const double4 s = frame_sums(a.acc, C, k, c);
                // E = sigma F: dE/dsigma = F, dE/dls = sigma H / ls
                g_sig += b.Eo * s.x + b.Ef * s.y;
                g_ls += (b.Eo * s.z + b.Ef * s.w) * a.sigma / a.ls;
                g_gam += b.g * a.gd[k];
                Fb = b.mf; Sb = b.ms; Db = b.md;
            }
        }
        g_pf += Fb;
        g_po += (Sb + Db) / 2.0;
    }
    double r;
    r = block_sum(loss * a.inv_n, sm);
    if (threadIdx.x == 0 && r != 0.0) atomicAdd(&a.red[0], r);
    if (!a.want_grad) return;
    r = block_sum(g_ls, sm);
    if (threadIdx.x == 0 && r != 0.0) atomicAdd(&a.red[1], r);
    r = block_sum(g_sig, sm);
    if (threadIdx.x == 0 && r != 0.0) atomicAdd(&a.red[2], r);
    r = block_sum(g_gam, sm);
    if (threadIdx.x == 0 && r != 0.0) atomicAdd(&a.red[3], r);
    r = block_sum(g_po, sm);
    if (threadIdx.x == 0 && r != 0.0) atomicAdd(&a.red[4], r);
    r = block_sum(g_pf, sm);
    if (threadIdx.x == 0 && r != 0.0) atomicAdd(&a.red[5], r);
}

// One frame's sums as four planes q x C (the layout k3dom_calib_get_sums returns).
__global__ void k_sums_planes(const long long* __restrict__ acc, long C, int k, double* __restrict__ out) {
    for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < C; c += (long)gridDim.x * blockDim.x) {
        const double4 v = frame_sums(acc, C, k, c);
        out[c] = v.x;
        out[C + c] = v.y;
        out[2 * C + c] = v.z;
        out[3 * C + c] = v.w;
    }
}

// ---------------------------------------------------------------- held-out labels (3-D DDA)
// Ray from the sensor s to the hit s + m, in continuous index space X = x / res + G / 2
// (cell i spans [i, i + 1)); Amanatides-Woo traversal in FP64 with the operations written out
// (no contraction), ties broken x before y before z. Every voxel before the hit voxel counts a
// free label (n0), the hit voxel a hit label (n1); voxels outside the grid are skipped.
struct DdaGrid {
    int G, Gz;
    double res;
};

__device__ inline void dda_ray(const DdaGrid& g, double sx, double sy, double sz, double mx, double my, double mz,
                               uint32_t* n0, uint32_t* n1) {
    const double half[3] = {g.G / 2.0, g.G / 2.0, g.Gz / 2.0};
    const int dims[3] = {g.G, g.G, g.Gz};
    const double a[3] = {__dadd_rn(__ddiv_rn(sx, g.res), half[0]), __dadd_rn(__ddiv_rn(sy, g.res), half[1]),
                         __dadd_rn(__ddiv_rn(sz, g.res), half[2])};
    const double b[3] = {__dadd_rn(__ddiv_rn(__dadd_rn(sx, mx), g.res), half[0]),
                         __dadd_rn(__ddiv_rn(__dadd_rn(sy, my), g.res), half[1]),
                         __dadd_rn(__ddiv_rn(__dadd_rn(sz, mz), g.res), half[2])};
    int v[3], e[3], step[3];
    double tmax[3], tdel[3];
    long budget = 1;
    for (int k = 0; k < 3; ++k) {
        v[k] = (int)floor(a[k]);
        e[k] = (int)floor(b[k]);
        const double d = __dsub_rn(b[k], a[k]);
        budget += abs(e[k] - v[k]);
        if (d > 0.0) {
            step[k] = 1;
            tdel[k] = __ddiv_rn(1.0, d);
            tmax[k] = __dmul_rn(__dsub_rn((double)(v[k] + 1), a[k]), tdel[k]);
        } else if (d < 0.0) {
            step[k] = -1;
            tdel[k] = __ddiv_rn(-1.0, d);
            tmax[k] = __dmul_rn(__dsub_rn(a[k], (double)v[k]), tdel[k]);
        } else {
            step[k] = 0;
            tdel[k] = INFINITY;
            tmax[k] = INFINITY;
        }
    }
    for (long it = 0; it < budget; ++it) {
        if (v[0] == e[0] && v[1] == e[1] && v[2] == e[2]) break;
        if (v[0] >= 0 && v[0] < dims[0] && v[1] >= 0 && v[1] < dims[1] && v[2] >= 0 && v[2] < dims[2])
            atomicAdd(&n0[v[0] + (long)g.G * v[1] + (long)g.G * g.G * v[2]], 1u);
        int k = 0;
        if (tmax[1] < tmax[k]) k = 1;
        if (tmax[2] < tmax[k]) k = 2;
        v[k] += step[k];
        tmax[k] = __dadd_rn(tmax[k], tdel[k]);
    }
    if (e[0] >= 0 && e[0] < dims[0] && e[1] >= 0 && e[1] < dims[1] && e[2] >= 0 && e[2] < dims[2])
        atomicAdd(&n1[e[0] + (long)g.G * e[1] + (long)g.G * g.G * e[2]], 1u);
}

__global__ void k_dda_labels(DdaGrid g, float sx, float sy, float sz, const float* __restrict__ xyz, int n,
                             uint32_t* n0, uint32_t* n1) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float mx = xyz[3 * i], my = xyz[3 * i + 1], mz = xyz[3 * i + 2];
        if (!(isfinite(mx) && isfinite(my) && isfinite(mz))) continue;
        dda_ray(g, sx, sy, sz, mx, my, mz, n0, n1);
    }
}

// xyz interleaved -> SoA
__global__ void k_split_xyz(const float* __restrict__ xyz, int n, float* x, float* y, float* z) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        x[i] = xyz[3 * i];
        y[i] = xyz[3 * i + 1];
        z[i] = xyz[3 * i + 2];
    }
}

struct CalibFrame {
    float dt;
    float sensor[3];
    int n;
    float* pts;  // device x | y | z
    float* dyn;  // device, C floats, or nullptr
};

}  // namespace

struct k3dom_calib {
    int device = 0, num_sms = 148;
    k3dom_params base{};
    DevParams dp{};
    cudaStream_t st = nullptr;
    std::vector<CalibFrame> frames;
    std::vector<void*> allocs, ray_allocs;
    uint32_t *n0 = nullptr, *n1 = nullptr;
    double n_labels = 0.0;
    SceneDev* sc_dev = nullptr;
    SceneOffsets* off_dev = nullptr;
    FrameParams* fp_dev = nullptr;  // one per frame
    // two lanes: frame k bins and sums on lane k % 2 (its own ray buffers, status and stream),
    // so one frame's ray lists are built while the other frame's sums run
    static constexpr int kLanes = 2;
    DevStatus* status = nullptr;  // kLanes entries
    RayBuffers rb[kLanes]{};
    cudaStream_t st2 = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    int ray_points = 0;
    float ray_ls = 0.0f;  // length-scale the list capacity was sized for
    float4 *ftab = nullptr, *htab = nullptr;
    long long* acc = nullptr;        // F x C x 4 exact unit sums of the frames
    double* sums_out = nullptr;      // 4 x C staging of k3dom_calib_get_sums
    int sums_frames = 0;
    double* red = nullptr;
    double red_host[6] = {0};
    float sums_ls = -1.0f;  // ls of the sums currently held
    cudaError_t last = cudaSuccess;

    k3dom_status fail(cudaError_t e) {
        last = e;
        return e == cudaErrorMemoryAllocation ? K3DOM_ERR_OUT_OF_MEMORY : K3DOM_ERR_CUDA;
    }
    template <typename T>
    cudaError_t alloc(T** p, size_t count, std::vector<void*>* list = nullptr) {
        *p = nullptr;
        cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(count, 1) * sizeof(T));
        if (e != cudaSuccess) return e;
        (list ? list : &allocs)->push_back((void*)*p);
        // on the problem's (non-blocking) stream, so it is ordered before the work that uses it
        return cudaMemsetAsync(*p, 0, std::max<size_t>(count, 1) * sizeof(T), st);
    }
    void release() {
        for (void* p : ray_allocs) cudaFree(p);
        for (void* p : allocs) cudaFree(p);
        ray_allocs.clear();
        allocs.clear();
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (st2) cudaStreamDestroy(st2);
        if (st) cudaStreamDestroy(st);
    }
};

namespace {

TileShape calib_tiles(const DevParams& p) {
    TileShape t;
    const bool large = (long)p.C >= (1L << 20) && p.Gz >= 8;
    t.tx = large ? 16 : 8;
    t.ty = large ? 16 : 8;
    t.tz = 4;
    t.ntx = (p.G + t.tx - 1) / t.tx;
    t.nty = (p.G + t.ty - 1) / t.ty;
    t.ntz = (p.Gz + t.tz - 1) / t.tz;
    t.nsbx = t.tx / 4;
    t.nsby = t.ty / 4;
    return t;
}

cudaError_t alloc_ray_lane(k3dom_calib* c, RayBuffers& rb, int max_points, long need, int T);

// Ray buffers for the largest frame at the scene's length-scale: re-made only when the point
// count or the worst-case list length outgrows them, then with 25 % headroom, so a calibration
// loop that moves ls a little does not reallocate.
cudaError_t ensure_ray_buffers(k3dom_calib* c, int max_points, float ls, const SceneDev& sd) {
    const int T = sd.ts.ntx * sd.ts.nty * sd.ts.ntz;
    long need = std::max(ray_entries_bound(sd.p, sd.ts, std::max(max_points, 1), sd.bin_R), 4096L);
    if (need > 0xFFFFFFF0L) need = 0xFFFFFFF0L;
    if (max_points <= c->ray_points && need <= c->rb[0].capacity && c->rb[0].evals2) return cudaSuccess;
    for (void* p : c->ray_allocs) cudaFree(p);
    c->ray_allocs.clear();
    for (int l = 0; l < k3dom_calib::kLanes; ++l) {
        cudaError_t e = alloc_ray_lane(c, c->rb[l], max_points, need, T);
        if (e != cudaSuccess) return e;
    }
    c->ray_points = std::max(max_points, 1);
    c->ray_ls = ls;
    return cudaSuccess;
}

cudaError_t alloc_ray_lane(k3dom_calib* c, RayBuffers& rb, int max_points, long need, int T) {
    rb = RayBuffers{};
    const int N = std::max(max_points, 1);
    long cap = std::min(need + need / 4, 0xFFFFFFF0L);
    rb.capacity = cap;
    rb.chunk = kCalibChunk;
    std::vector<void*>* L = &c->ray_allocs;
    cudaError_t e;
    if ((e = c->alloc(&rb.ray_a, N, L)) || (e = c->alloc(&rb.ray_c, N, L)) ||
        (e = c->alloc(&rb.counts, (size_t)kRayThreads * N, L)) ||
        (e = c->alloc(&rb.evals2, cap, L)) || (e = c->alloc(&rb.tile_start, T + 1, L)) ||
        (e = c->alloc(&rb.item_off, T + 1, L)) || (e = c->alloc(&rb.tile_done, T, L)) || (e = c->alloc(&rb.total, 4, L)))
        return e;
    if (placed_lists(false, T))  // lists placed per tile through tallies and per-block offsets
        return (e = c->alloc(&rb.tile_tally, T, L))
                   ? e
                   : c->alloc(&rb.block_base, (size_t)bin_blocks((long)kRayThreads * N) * T, L);
    // lists sorted by tile
    if ((e = c->alloc(&rb.offsets, N, L)) || (e = c->alloc(&rb.ekeys, cap, L)) || (e = c->alloc(&rb.evals, cap, L)) ||
        (e = c->alloc(&rb.ekeys2, cap, L)) || (e = c->alloc(&rb.tile_items, T, L)))
        return e;
    int bits = 1;
    while ((1 << bits) < T + 1) ++bits;
    int pb[8];
    if (onesweep_plan(bits, pb) > 1) {
        if ((e = c->alloc(&rb.ekeys_alt, cap, L)) || (e = c->alloc(&rb.evals_alt, cap, L))) return e;
    } else {
        rb.ekeys_alt = rb.ekeys;
        rb.evals_alt = rb.evals;
    }
    rb.os_words = onesweep_scratch_words(cap, bits);
    rb.scan_words = scan_u32_tiles(std::max((long)N, (long)T + 1)) + 16;
    if ((e = c->alloc(&rb.os_scratch, rb.os_words, L)) || (e = c->alloc(&rb.scan_tmp, rb.scan_words, L))) return e;
    return cudaSuccess;
}

// The per-frame kernel and derivative sums at length-scale ls (kept until ls changes).
k3dom_status compute_sums(k3dom_calib* c, float ls) {
    const int F = (int)c->frames.size();
    if (F == 0) return K3DOM_ERR_NOT_READY;
    if (ls == c->sums_ls && c->sums_frames == F) return K3DOM_OK;
    cudaError_t e;
    const long C = c->dp.C;
    if (c->sums_frames != F) {
        if (c->acc) {
            auto it = std::find(c->allocs.begin(), c->allocs.end(), (void*)c->acc);
            if (it != c->allocs.end()) c->allocs.erase(it);
            cudaFree(c->acc);
            c->acc = nullptr;
        }
        if ((e = c->alloc(&c->acc, (size_t)F * 4 * C))) return c->fail(e);
        c->sums_frames = F;
    }
    SceneDev sd;
    std::memset(&sd, 0, sizeof(sd));
    sd.p = c->dp;
    sd.p.ls = ls;
    sd.p.sigma = 1.0f;
    sd.ts = calib_tiles(sd.p);
    sd.n_tiles = sd.ts.ntx * sd.ts.nty * sd.ts.ntz;
    fill_scene_evidence(sd, false, nullptr);
    int maxn = 0;
    for (auto& f : c->frames) maxn = std::max(maxn, f.n);
    if ((e = ensure_ray_buffers(c, maxn, ls, sd))) return c->fail(e);
    sd.max_points = c->ray_points;
    if ((e = cudaMemcpyAsync(c->sc_dev, &sd, sizeof(sd), cudaMemcpyHostToDevice, c->st))) return c->fail(e);
    for (int k = 0; k < F; ++k) {
        const CalibFrame& f = c->frames[k];
        SceneOffsets off;
        std::memset(&off, 0, sizeof(off));
        off.point[1] = f.n;
        off.tile[1] = sd.n_tiles;
        off.cell[1] = (int)C;
        off.part[1] = c->dp.P;
        off.birth[1] = c->dp.B;
        off.joint[1] = c->dp.P + c->dp.B;
        FrameParams fp;
        std::memset(&fp, 0, sizeof(fp));
        fp.dt = f.dt;
        fp.sensor_x = f.sensor[0];
        fp.sensor_y = f.sensor[1];
        fp.sensor_z = f.sensor[2];
        fp.n_points = f.n;
        if ((e = cudaMemcpyAsync(c->off_dev + k, &off, sizeof(off), cudaMemcpyHostToDevice, c->st)) ||
            (e = cudaMemcpyAsync(c->fp_dev + k, &fp, sizeof(fp), cudaMemcpyHostToDevice, c->st)))
            return c->fail(e);
    }
    if ((e = cudaEventRecord(c->ev_fork, c->st)) || (e = cudaStreamWaitEvent(c->st2, c->ev_fork, 0)))
        return c->fail(e);
    for (int k = 0; k < F; ++k) {
        const CalibFrame& f = c->frames[k];
        const int l = k % k3dom_calib::kLanes;
        cudaStream_t sk = l == 0 ? c->st : c->st2;
        Batch bt;
        bt.S = 1;
        bt.variant = 0;
        bt.P = c->dp.P;
        bt.B = c->dp.B;
        bt.C = (int)C;
        bt.N = f.n;
        bt.T = sd.n_tiles;
        bt.sc = c->sc_dev;
        bt.fp = c->fp_dev + k;
        bt.off = c->off_dev + k;
        long long* acc_k = c->acc + (long)k * 4 * C;
        if ((e = cudaMemsetAsync(acc_k, 0, sizeof(long long) * 4 * (size_t)C, sk))) return c->fail(e);
        if (f.n > 0) {
            if ((e = build_ray_lists(bt, f.pts, f.pts + f.n, f.pts + 2 * (long)f.n, c->rb[l], false, c->status + l,
                                     SortWait(), sk)))
                return c->fail(e);
            if ((e = launch_bgki_sums(bt, c->rb[l], c->ftab, c->htab, reinterpret_cast<unsigned long long*>(acc_k),
                                      c->status + l, c->num_sms, sk)))
                return c->fail(e);
        }
    }
    if ((e = cudaEventRecord(c->ev_join, c->st2)) || (e = cudaStreamWaitEvent(c->st, c->ev_join, 0)))
        return c->fail(e);
    DevStatus dst[k3dom_calib::kLanes];
    if ((e = cudaMemcpyAsync(dst, c->status, sizeof(dst), cudaMemcpyDeviceToHost, c->st)) ||
        (e = cudaStreamSynchronize(c->st)))
        return c->fail(e);
    for (int l = 0; l < k3dom_calib::kLanes; ++l) {
        if (dst[l].sort_timeout) return K3DOM_ERR_TIMEOUT;  // a bounded wait of the ray-list sort gave up
        if (dst[l].overflow) return K3DOM_ERR_CAPACITY;
    }
    c->sums_ls = ls;
    return K3DOM_OK;
}

k3dom_status run_cells(k3dom_calib* c, const float theta[5], bool grad, float* occ_out) {
    if (!(theta[0] > 0.0f) || !(theta[2] > 0.0f)) return K3DOM_ERR_INVALID_ARGUMENT;
    if (c->n_labels <= 0.0 && !occ_out) return K3DOM_ERR_NOT_READY;
    k3dom_status s = compute_sums(c, theta[0]);
    if (s != K3DOM_OK) return s;
    CalibCellArgs a;
    std::memset(&a, 0, sizeof(a));
    a.C = c->dp.C;
    a.F = (int)c->frames.size();
    a.ls = theta[0];
    a.sigma = theta[1];
    a.gamma = theta[2];
    a.prior_occ = theta[3];
    a.prior_free = theta[4];
    a.k2 = 2.0 / (double)c->dp.mass_scale;
    a.inv_n = c->n_labels > 0.0 ? 1.0 / c->n_labels : 0.0;
    for (int k = 0; k < a.F; ++k) {
        const double dt = c->frames[k].dt;
        a.g[k] = k == 0 ? 1.0 : std::pow(a.gamma, dt);
        a.gd[k] = (k > 0 && dt > 0.0) ? dt * std::pow(a.gamma, dt - 1.0) : 0.0;
        a.dyn[k] = c->frames[k].dyn;
    }
    a.acc = c->acc;
    a.n0 = c->n0;
    a.n1 = c->n1;
    a.occ_out = occ_out;
    a.red = c->red;
    a.want_grad = grad ? 1 : 0;
    cudaError_t e;
    if ((e = cudaMemsetAsync(c->red, 0, 6 * sizeof(double), c->st))) return c->fail(e);
    ++g_launches;
    // one wave of resident blocks: each block reduces its partial sums once, at the end
    auto kern = a.F <= 2 ? k_calib_cells<2> : a.F <= 4 ? k_calib_cells<4> : k_calib_cells<kMaxCalibFrames>;
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0);
    const long blocks = std::min<long>((long)c->num_sms * std::max(1, per_sm), (a.C + 255) / 256);
    kern<<<(unsigned)std::max(1L, blocks), 256, 0, c->st>>>(a);
    if ((e = cudaGetLastError()) || (e = cudaMemcpyAsync(c->red_host, c->red, 6 * sizeof(double),
                                                         cudaMemcpyDeviceToHost, c->st)) ||
        (e = cudaStreamSynchronize(c->st)))
        return c->fail(e);
    return K3DOM_OK;
}

cudaError_t to_device_copy(k3dom_calib* c, float** dst, const float* src, size_t count, k3dom_mem mem) {
    cudaError_t e = c->alloc(dst, count);
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(*dst, src, count * sizeof(float),
                           mem == K3DOM_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, c->st);
}

}  // namespace

extern "C" {

k3dom_status k3dom_calib_create(const k3dom_params* base, int device, k3dom_calib** out) {
    if (!out || !base) return K3DOM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (!(base->resolution > 0.0f) || !(base->size > 0.0f) || !(base->size_z > 0.0f) || !(base->mass_scale != 0.0f))
        return K3DOM_ERR_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return K3DOM_ERR_NO_DEVICE;
    if (device < 0 || device >= ndev) return K3DOM_ERR_INVALID_ARGUMENT;
    k3dom_calib* c = new (std::nothrow) k3dom_calib();
    if (!c) return K3DOM_ERR_OUT_OF_MEMORY;
    auto bail = [&](cudaError_t e) {
        k3dom_status r = c->fail(e);
        c->release();
        delete c;
        return r;
    };
    c->device = device;
    c->base = *base;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return bail(e);
    cudaDeviceProp prop;
    if ((e = cudaGetDeviceProperties(&prop, device))) return bail(e);
    c->num_sms = prop.multiProcessorCount;
    if ((e = sort_init()) || (e = evidence_init())) return bail(e);
    DevParams& d = c->dp;
    d.G = static_cast<int>(base->size / base->resolution);
    d.Gz = static_cast<int>(base->size_z / base->resolution);
    if (d.G < 1 || d.Gz < 1 || (double)d.G * d.G * d.Gz > 2147483647.0 / 4) return bail(cudaErrorInvalidValue);
    d.C = d.G * d.G * d.Gz;
    d.P = 1;
    d.B = 1;
    d.res = base->resolution;
    d.size = base->size;
    d.size_z = base->size_z;
    d.mass_scale = base->mass_scale;
    d.ls = base->ls;
    d.sigma = 1.0f;
    d.window_radius = base->resolution * 0.866f;
    if ((e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking)) ||
        (e = cudaStreamCreateWithFlags(&c->st2, cudaStreamNonBlocking)) ||
        (e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming)) ||
        (e = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming)))
        return bail(e);
    if ((e = c->alloc(&c->n0, d.C)) || (e = c->alloc(&c->n1, d.C)) || (e = c->alloc(&c->sc_dev, 1)) ||
        (e = c->alloc(&c->off_dev, kMaxCalibFrames)) || (e = c->alloc(&c->fp_dev, kMaxCalibFrames)) ||
        (e = c->alloc(&c->status, k3dom_calib::kLanes)) || (e = c->alloc(&c->ftab, kKernelTableSize)) ||
        (e = c->alloc(&c->htab, kKernelTableSize)) || (e = c->alloc(&c->sums_out, 4 * (size_t)d.C)) ||
        (e = c->alloc(&c->red, 6)))
        return bail(e);
    std::vector<float4> ft(kKernelTableSize), ht(kKernelTableSize);
    build_calib_tables(ft.data(), ht.data());
    if ((e = cudaMemcpyAsync(c->ftab, ft.data(), sizeof(float4) * ft.size(), cudaMemcpyHostToDevice, c->st)) ||
        (e = cudaMemcpyAsync(c->htab, ht.data(), sizeof(float4) * ht.size(), cudaMemcpyHostToDevice, c->st)) ||
        (e = cudaStreamSynchronize(c->st)))
        return bail(e);
    *out = c;
    return K3DOM_OK;
}

k3dom_status k3dom_calib_destroy(k3dom_calib* c) {
    if (!c) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->st);
    c->release();
    delete c;
    return K3DOM_OK;
}

k3dom_status k3dom_calib_add_frame(k3dom_calib* c, float dt, float sx, float sy, float sz, const float* xyz,
                                   int32_t n, const float* dyn_pred, k3dom_mem mem) {
    if (!c || n < 0 || (n > 0 && !xyz) || !(dt >= 0.0f)) return K3DOM_ERR_INVALID_ARGUMENT;
    if ((int)c->frames.size() >= kMaxCalibFrames) return K3DOM_ERR_CAPACITY;
    if (c->frames.empty() && dt != 0.0f) return K3DOM_ERR_INVALID_ARGUMENT;  // frame 0 initialises
    if (mem == K3DOM_MEM_HOST)
        for (long i = 0; i < 3L * n; ++i)
            if (!std::isfinite(xyz[i])) return K3DOM_ERR_INVALID_INPUT;
    cudaSetDevice(c->device);
    CalibFrame f;
    f.dt = dt;
    f.sensor[0] = sx;
    f.sensor[1] = sy;
    f.sensor[2] = sz;
    f.n = n;
    f.pts = nullptr;
    f.dyn = nullptr;
    cudaError_t e;
    float* tmp = nullptr;
    if ((e = c->alloc(&f.pts, 3 * (size_t)std::max(n, 1)))) return c->fail(e);
    if (n > 0) {
        if ((e = to_device_copy(c, &tmp, xyz, 3 * (size_t)n, mem))) return c->fail(e);
        ++g_launches;
        k_split_xyz<<<grid_for(n), kBlock, 0, c->st>>>(tmp, n, f.pts, f.pts + n, f.pts + 2 * (long)n);
        if ((e = cudaGetLastError())) return c->fail(e);
    }
    if (dyn_pred && (e = to_device_copy(c, &f.dyn, dyn_pred, (size_t)c->dp.C, mem))) return c->fail(e);
    if ((e = cudaStreamSynchronize(c->st))) return c->fail(e);
    if (tmp) {
        auto it = std::find(c->allocs.begin(), c->allocs.end(), (void*)tmp);
        if (it != c->allocs.end()) c->allocs.erase(it);
        cudaFree(tmp);
    }
    c->frames.push_back(f);
    c->sums_ls = -1.0f;
    return K3DOM_OK;
}

k3dom_status k3dom_calib_add_heldout_scan(k3dom_calib* c, float sx, float sy, float sz, const float* xyz, int32_t n,
                                          k3dom_mem mem) {
    if (!c || n < 0 || (n > 0 && !xyz)) return K3DOM_ERR_INVALID_ARGUMENT;
    if (n == 0) return K3DOM_OK;
    cudaSetDevice(c->device);
    cudaError_t e;
    float* tmp = nullptr;
    const float* src = xyz;
    if (mem == K3DOM_MEM_HOST) {
        if ((e = to_device_copy(c, &tmp, xyz, 3 * (size_t)n, mem))) return c->fail(e);
        src = tmp;
    }
    DdaGrid g;
    g.G = c->dp.G;
    g.Gz = c->dp.Gz;
    g.res = c->dp.res;
    ++g_launches;
    k_dda_labels<<<grid_for(n), kBlock, 0, c->st>>>(g, sx, sy, sz, src, n, c->n0, c->n1);
    if ((e = cudaGetLastError()) || (e = cudaStreamSynchronize(c->st))) return c->fail(e);
    if (tmp) {
        auto it = std::find(c->allocs.begin(), c->allocs.end(), (void*)tmp);
        if (it != c->allocs.end()) c->allocs.erase(it);
        cudaFree(tmp);
    }
    // total label instances
    std::vector<uint32_t> h0(c->dp.C), h1(c->dp.C);
    if ((e = cudaMemcpyAsync(h0.data(), c->n0, sizeof(uint32_t) * h0.size(), cudaMemcpyDeviceToHost, c->st)) ||
        (e = cudaMemcpyAsync(h1.data(), c->n1, sizeof(uint32_t) * h1.size(), cudaMemcpyDeviceToHost, c->st)) ||
        (e = cudaStreamSynchronize(c->st)))
        return c->fail(e);
    double tot = 0.0;
    for (size_t i = 0; i < h0.size(); ++i) tot += (double)h0[i] + (double)h1[i];
    c->n_labels = tot;
    return K3DOM_OK;
}

k3dom_status k3dom_calib_label_counts(k3dom_calib* c, uint32_t* n0, uint32_t* n1, k3dom_mem mem) {
    if (!c) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    const cudaMemcpyKind k = mem == K3DOM_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    cudaError_t e = cudaSuccess;
    if (n0) e = cudaMemcpyAsync(n0, c->n0, sizeof(uint32_t) * (size_t)c->dp.C, k, c->st);
    if (e == cudaSuccess && n1) e = cudaMemcpyAsync(n1, c->n1, sizeof(uint32_t) * (size_t)c->dp.C, k, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    return e == cudaSuccess ? K3DOM_OK : c->fail(e);
}

k3dom_status k3dom_calib_get_sums(k3dom_calib* c, float ls, int32_t frame, double* out, k3dom_mem mem) {
    if (!c || !out || frame < 0 || frame >= (int)c->frames.size() || !(ls > 0.0f)) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    k3dom_status s = compute_sums(c, ls);
    if (s != K3DOM_OK) return s;
    const size_t C = (size_t)c->dp.C;
    double* planes = mem == K3DOM_MEM_HOST ? c->sums_out : out;
    ++g_launches;
    k_sums_planes<<<grid_for((long)C), kBlock, 0, c->st>>>(c->acc, (long)C, frame, planes);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && mem == K3DOM_MEM_HOST)
        e = cudaMemcpyAsync(out, planes, sizeof(double) * 4 * C, cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    return e == cudaSuccess ? K3DOM_OK : c->fail(e);
}

k3dom_status k3dom_bgki_forward(k3dom_calib* c, const float* theta, float* loss, float* occupancy, k3dom_mem mem) {
    if (!c || !theta) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    float* occ_dev = nullptr;
    cudaError_t e;
    if (occupancy) {
        if (mem == K3DOM_MEM_DEVICE) {
            occ_dev = occupancy;
        } else if ((e = c->alloc(&occ_dev, (size_t)c->dp.C))) {
            return c->fail(e);
        }
    }
    k3dom_status s = run_cells(c, theta, false, occ_dev);
    if (s == K3DOM_OK && occupancy && mem == K3DOM_MEM_HOST) {
        e = cudaMemcpyAsync(occupancy, occ_dev, sizeof(float) * (size_t)c->dp.C, cudaMemcpyDeviceToHost, c->st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
        if (e != cudaSuccess) s = c->fail(e);
    }
    if (occupancy && mem == K3DOM_MEM_HOST && occ_dev) {
        auto it = std::find(c->allocs.begin(), c->allocs.end(), (void*)occ_dev);
        if (it != c->allocs.end()) c->allocs.erase(it);
        cudaFree(occ_dev);
    }
    if (s == K3DOM_OK && loss) *loss = (float)c->red_host[0];
    return s;
}

k3dom_status k3dom_bgki_backward(k3dom_calib* c, const float* theta, float grad_loss, float* grad_theta,
                                 float* loss) {
    if (!c || !theta || !grad_theta) return K3DOM_ERR_INVALID_ARGUMENT;
    cudaSetDevice(c->device);
    k3dom_status s = run_cells(c, theta, true, nullptr);
    if (s != K3DOM_OK) return s;
    for (int i = 0; i < 5; ++i) grad_theta[i] = (float)(grad_loss * c->red_host[1 + i]);
    if (loss) *loss = (float)c->red_host[0];
    return K3DOM_OK;
}

k3dom_status k3dom_calib_info(k3dom_calib* c, int32_t* cells, int32_t* frames, double* label_instances) {
    if (!c) return K3DOM_ERR_INVALID_ARGUMENT;
    if (cells) *cells = c->dp.C;
    if (frames) *frames = (int32_t)c->frames.size();
    if (label_instances) *label_instances = c->n_labels;
    return K3DOM_OK;
}

k3dom_status k3dom_calib_get_stream(k3dom_calib* c, void** stream) {
    if (!c || !stream) return K3DOM_ERR_INVALID_ARGUMENT;
    *stream = (void*)c->st;
    return K3DOM_OK;
}

}  // extern "C"
