/*
 * k3dom_oracle.c -- TEST INFRASTRUCTURE ONLY. A CPU restatement of the reference's
 * per-frame update (youngjae-min/k3dom), used by the tests, by smoke() and by the benchmark's
 * CPU-baseline leg as the checker. No product code path calls it.
 *
 * Precision model
 *  - Continuous outputs (BGKI evidence, masses, mean velocities, reweighted weights) are
 *    evaluated in FP64 from the same FP32 inputs; the GPU must agree within a relative
 *    tolerance.
 *  - Discrete outputs (voxel indices, sort order, birth slots, ancestors, DS neighbour sets)
 *    are restated in FP32 with the reference's operation order (this file is compiled with
 *    -ffp-contract=off, so every float operation rounds once, as the GPU code does with _rn
 *    intrinsics and as the reference does when built with -fmad=false).
 *  - The two scans whose results decide integers (born masses -> birth slots, joint weights
 *    -> ancestors) are exact: floats are summed as 128-bit fixed-point integers (2^-80
 *    resolution) and each prefix is rounded once to float.
 * Citations are file:line in the reference repository.
 */
#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------ draws (Philox4x32-10) */
typedef struct { uint32_t x, y, z, w; } U4;

static U4 philox(U4 c, uint32_t k0, uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)M0 * c.x, p1 = (uint64_t)M1 * c.z;
        U4 n;
        n.x = (uint32_t)(p1 >> 32) ^ c.y ^ k0;
        n.y = (uint32_t)p1;
        n.z = (uint32_t)(p0 >> 32) ^ c.w ^ k1;
        n.w = (uint32_t)p0;
        c = n;
        k0 += W0;
        k1 += W1;
    }
    return c;
}

static U4 draw_block(uint64_t seed, uint32_t frame, uint32_t stage, uint64_t item, uint32_t blk) {
    U4 c = {(uint32_t)item, (uint32_t)(item >> 32), blk | (stage << 24), frame};
    return philox(c, (uint32_t)seed, (uint32_t)(seed >> 32));
}
static float u01(uint32_t r) { return (float)((r >> 8) + 1u) * 5.9604644775390625e-08f; }
static uint32_t pick(U4 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w)); }

/* Raw Philox4x32-10 block (for the published known-answer vectors). */
void orc_philox_raw(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
    U4 c = {ctr[0], ctr[1], ctr[2], ctr[3]};
    U4 r = philox(c, key[0], key[1]);
    out[0] = r.x;
    out[1] = r.y;
    out[2] = r.z;
    out[3] = r.w;
}

/* Uniform draws: stage 2/3 -> 3 per item, stage 4 -> 1 per item. */
void orc_uniforms(uint64_t seed, uint32_t frame, uint32_t stage, int64_t first, int64_t count, float* out) {
    for (int64_t t = 0; t < count; ++t) {
        uint64_t it = (uint64_t)(first + t);
        if (stage == 4) {
            out[t] = u01(pick(draw_block(seed, frame, 4, it >> 2, 0), (int)(it & 3)));
        } else {
            U4 b = draw_block(seed, frame, stage, it, 0);
            out[3 * t] = u01(b.x);
            out[3 * t + 1] = u01(b.y);
            out[3 * t + 2] = u01(b.z);
        }
    }
}

/* Resampling sort keys: 1 - u on the 2^-24 grid. */
void orc_resample_keys(uint64_t seed, uint32_t frame, int64_t count, uint32_t* out) {
    for (int64_t i = 0; i < count; ++i)
        out[i] = 0xFFFFFFu - (pick(draw_block(seed, frame, 4, (uint64_t)i >> 2, 0), (int)(i & 3)) >> 8);
}

/* Prediction normals with libm (not bit-equal to the GPU's; CPU-only runs). */
void orc_normals_libm(uint64_t seed, uint32_t frame, int64_t first, int64_t count, float* out) {
    for (int64_t t = 0; t < count; ++t) {
        uint64_t it = (uint64_t)(first + t);
        for (int k = 0; k < 6; ++k) {
            U4 b = draw_block(seed, frame, 1, it, (uint32_t)(k >> 2));
            int p = (k & 3) >> 1;
            float u1 = u01(pick(b, 2 * p)), u2 = u01(pick(b, 2 * p + 1));
            double rho = sqrt(-2.0 * log((double)u1));
            double th = 2.0 * M_PI * (double)u2;
            out[6 * t + k] = (float)((k & 1) ? rho * sin(th) : rho * cos(th));
        }
    }
}

/* ------------------------------------------------------------------ FP32 helpers */
/* cvt.rzi.s32.f32: truncate, saturate, NaN -> 0 */
static int f2i(float x) {
    if (x != x) return 0;
    if (x >= 2147483648.0f) return INT_MAX;
    if (x <= -2147483648.0f) return INT_MIN;
    return (int)x;
}
static int clampi(int a, int lo, int hi) { return a < lo ? lo : (a > hi ? hi : a); }
static float clampf(float a, float lo, float hi) { return fmaxf(fminf(a, hi), lo); }

/* ------------------------------------------------------------------ prediction */
/* predictKernel (src/common/kernel/predict.cu:12-59), with moveParticlesKernel
 * (ego_motion_compensation.cu:12-18) applied first when a shift is pending. normals holds
 * the 6 draws per particle (pos x,y,z, vel x,y,z). */
void orc_predict(int n, int G, int Gz, float dt, float p_S, float noise_pos, float noise_vel, float imv,
                 int shift_pending, int sx, int sy, int sz, const float* normals, float* px, float* py, float* pz,
                 float* vx, float* vy, float* vz, float* w, int32_t* cell) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        float x = px[i], y = py[i], z = pz[i], a = vx[i], b = vy[i], c = vz[i], ww = w[i];
        if (shift_pending) {
            x = x - (float)sx;
            y = y - (float)sy;
            z = z - (float)sz;
        }
        const float* nn = normals + 6 * (int64_t)i;
        float npx = nn[0] * noise_pos + 0.0f, npy = nn[1] * noise_pos + 0.0f, npz = nn[2] * noise_pos + 0.0f;
        float nvx = nn[3] * noise_vel + 0.0f, nvy = nn[4] * noise_vel + 0.0f, nvz = nn[5] * noise_vel + 0.0f;
        float tx = a * dt, ty = b * dt, tz = c * dt;
        tx = tx + npx;
        ty = ty + npy;
        tz = tz + npz;
        x = x + tx;
        y = y + ty;
        z = z + tz;
        a = a + nvx;
        b = b + nvy;
        c = c + nvz;
        ww = ww * p_S;
        float lim = 5.0f * imv, nlim = -5.0f * imv;
        a = clampf(a, nlim, lim);
        b = clampf(b, nlim, lim);
        c = clampf(c, nlim, lim);
        if ((x >= (float)G || x < 0.0f) || (y >= (float)G || y < 0.0f) || (z >= (float)Gz || z < 0.0f)) ww = 0.0f;
        int ix = clampi(f2i(x), 0, G - 1), iy = clampi(f2i(y), 0, G - 1), iz = clampi(f2i(z), 0, Gz - 1);
        px[i] = x; py[i] = y; pz[i] = z;
        vx[i] = a; vy[i] = b; vz[i] = c;
        w[i] = ww;
        cell[i] = ix + G * iy + G * G * iz;
    }
}

/* ------------------------------------------------------------------ assignment */
/* thrust::sort_by_key on the cell keys (src/common/dom.cu:175-183) is a stable sort:
 * restated as a stable counting sort. particleToGridKernel ranges (particle_to_grid.cu). */
void orc_assign(int n, int C, const int32_t* keys, int32_t* perm, int32_t* sorted_keys, int32_t* start, int32_t* end) {
    int64_t* cnt = (int64_t*)calloc((size_t)C + 1, sizeof(int64_t));
    for (int i = 0; i < n; ++i) cnt[keys[i] + 1]++;
    for (int c = 0; c < C; ++c) cnt[c + 1] += cnt[c];
    for (int i = 0; i < n; ++i) {
        int64_t pos = cnt[keys[i]]++;
        perm[pos] = i;
        sorted_keys[pos] = keys[i];
    }
    for (int c = 0; c < C; ++c) start[c] = end[c] = -1;
    for (int i = 0; i < n; ++i) {
        int k = sorted_keys[i];
        if (i == 0 || sorted_keys[i - 1] != k) start[k] = i;
        if (i == n - 1 || sorted_keys[i + 1] != k) end[k] = i;
    }
    free(cnt);
}

/* Per-cell sums over a sorted set: sum w (the loop of mass_update.cu:168-174) and sum w*v
 * with w*v rounded to float as statisticalMomentsKernel1 stores it. */
void orc_cell_sums(int n, int C, const int32_t* skeys, const float* w, const float* vx, const float* vy,
                   const float* vz, double* sw, double* swx, double* swy, double* swz) {
    for (int c = 0; c < C; ++c) sw[c] = swx[c] = swy[c] = swz[c] = 0.0;
    for (int i = 0; i < n; ++i) {
        int c = skeys[i];
        float ww = fabsf(w[i]);
        sw[c] += ww;
        swx[c] += (double)(ww * vx[i]);
        swy[c] += (double)(ww * vy[i]);
        swz[c] += (double)(ww * vz[i]);
    }
}

/* ------------------------------------------------------------------ geometry */
typedef struct {
    int G, Gz;
    float res, sx, sy, sz; /* sensor minus map centre [m] */
} orc_grid;

/* cell centre relative to the sensor in FP32, reference order (mass_update.cu:92-99) */
static void centre_f(const orc_grid* g, int ix, int iy, int iz, float* x, float* y, float* z) {
    float hg = (float)g->G / 2.0f, hz = (float)g->Gz / 2.0f;
    float a = (float)ix + 0.5f, b = (float)iy + 0.5f, c = (float)iz + 0.5f;
    a = a - hg; b = b - hg; c = c - hz;
    a = a * g->res; b = b * g->res; c = c * g->res;
    *x = a - g->sx;
    *y = b - g->sy;
    *z = c - g->sz;
}

/* ------------------------------------------------------------------ BGKI (FP64) */
static double kernel_d(double d, double ls, double sigma) {
    /* mass_update.cu:24-26 */
    double x = d / ls;
    double v = sigma * ((2.0 + cos(M_PI * 2.0 * x)) * (1.0 - x) / 3.0 + sin(M_PI * 2.0 * x) / (2.0 * 3.141592));
    return v > 0.0 ? v : 0.0;
}

/* Evidence of one (cell, point) pair, exactly the branches of BGKI (mass_update.cu:43-71).
 * tie gets the free contribution that a float-level flip of d_proj < d_m would toggle. */
static void bgki_pair(double cx, double cy, double cz, double mx, double my, double mz, double res, double ls,
                      double sigma, double* occ, double* fr, double* tie, int* ntie) {
    double dx = cx - mx, dy = cy - my, dz = cz - mz;
    double d = sqrt(dx * dx + dy * dy + dz * dz);
    if (d < ls) *occ += kernel_d(d, ls, sigma);
    double dc = sqrt(cx * cx + cy * cy + cz * cz);
    double dm = sqrt(mx * mx + my * my + mz * mz);
    if (!(dm > 0.0)) return; /* 0/0 in the reference: every comparison false -> no free */
    double dp = (cx * mx + cy * my + cz * mz) / dm;
    double marg = fmax(0.9 * dm, dm - 2.0 * res);
    double df;
    if (dp <= 0.0) {
        df = dc;
    } else if (dp < marg) {
        double q = dc * dc - dp * dp;
        df = sqrt(q > 0.0 ? q : 0.0);
    } else {
        double r = marg / dm;
        double ex = cx - r * mx, ey = cy - r * my, ez = cz - r * mz;
        df = sqrt(ex * ex + ey * ey + ez * ez);
    }
    double kf = df < ls ? kernel_d(df, ls, sigma) : 0.0;
    if (fabs(dp - dm) <= 1e-6 * (1.0 + dm) && kf > 0.0) {
        *tie += kf;
        *ntie += 1;
    }
    if (dp < dm) *fr += kf;
}

/* Sparse BGKI over the grid: cells within ls of each point (occupied) and of each ray's
 * segment (free), enumerated by slabs along the ray's dominant axis; the same nonzero
 * terms as the reference's brute force over all (cell, point) pairs. */
void orc_bgki(const orc_grid* g, float ls, float sigma, int n, const float* xs, const float* ys, const float* zs,
              double* del_occ, double* del_free, double* tie_mass, int32_t* tie_count) {
    const int G = g->G, Gz = g->Gz;
    const int64_t C = (int64_t)G * G * Gz;
    memset(del_occ, 0, sizeof(double) * C);
    memset(del_free, 0, sizeof(double) * C);
    memset(tie_mass, 0, sizeof(double) * C);
    memset(tie_count, 0, sizeof(int32_t) * C);
    const double res = g->res;
    const double R = (double)ls / res + 1e-6;
    const double au[3] = {(double)g->sx / res + G / 2.0 - 0.5, (double)g->sy / res + G / 2.0 - 0.5,
                          (double)g->sz / res + Gz / 2.0 - 0.5};
    const int dims[3] = {G, G, Gz};
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
        const double m[3] = {xs[i], ys[i], zs[i]};
        if (!isfinite(m[0]) || !isfinite(m[1]) || !isfinite(m[2])) continue;
        const double bu[3] = {au[0] + m[0] / res, au[1] + m[1] / res, au[2] + m[2] / res};
        const double d[3] = {bu[0] - au[0], bu[1] - au[1], bu[2] - au[2]};
        int A = 0;
        if (fabs(d[1]) > fabs(d[A])) A = 1;
        if (fabs(d[2]) > fabs(d[A])) A = 2;
        const int Bx = (A + 1) % 3, Cx = (A + 2) % 3;
        int lo = (int)floor(fmin(au[A], bu[A]) - R), hi = (int)ceil(fmax(au[A], bu[A]) + R);
        if (lo < 0) lo = 0;
        if (hi > dims[A] - 1) hi = dims[A] - 1;
        for (int ia = lo; ia <= hi; ++ia) {
            double t0 = 0.0, t1 = 1.0;
            if (d[A] != 0.0) {
                double e0 = (ia - R - au[A]) / d[A], e1 = (ia + R - au[A]) / d[A];
                t0 = fmax(t0, fmin(e0, e1));
                t1 = fmin(t1, fmax(e0, e1));
                if (t0 > t1) continue;
            } else if (fabs(ia - au[A]) > R) {
                continue;
            }
            double b0 = au[Bx] + d[Bx] * t0, b1 = au[Bx] + d[Bx] * t1;
            double c0 = au[Cx] + d[Cx] * t0, c1 = au[Cx] + d[Cx] * t1;
            int ib0 = (int)floor(fmin(b0, b1) - R), ib1 = (int)ceil(fmax(b0, b1) + R);
            int ic0 = (int)floor(fmin(c0, c1) - R), ic1 = (int)ceil(fmax(c0, c1) + R);
            if (ib0 < 0) ib0 = 0;
            if (ic0 < 0) ic0 = 0;
            if (ib1 > dims[Bx] - 1) ib1 = dims[Bx] - 1;
            if (ic1 > dims[Cx] - 1) ic1 = dims[Cx] - 1;
            for (int ib = ib0; ib <= ib1; ++ib)
                for (int ic = ic0; ic <= ic1; ++ic) {
                    int idx3[3];
                    idx3[A] = ia;
                    idx3[Bx] = ib;
                    idx3[Cx] = ic;
                    float cxf, cyf, czf;
                    centre_f(g, idx3[0], idx3[1], idx3[2], &cxf, &cyf, &czf);
                    double oc = 0, of = 0, tm = 0;
                    int nt = 0;
                    bgki_pair(cxf, cyf, czf, m[0], m[1], m[2], res, ls, sigma, &oc, &of, &tm, &nt);
                    if (oc == 0.0 && of == 0.0 && nt == 0) continue;
                    int64_t c = idx3[0] + (int64_t)G * idx3[1] + (int64_t)G * G * idx3[2];
                    if (oc != 0.0) {
#pragma omp atomic
                        del_occ[c] += oc;
                    }
                    if (of != 0.0) {
#pragma omp atomic
                        del_free[c] += of;
                    }
                    if (nt) {
#pragma omp atomic
                        tie_mass[c] += tm;
#pragma omp atomic
                        tie_count[c] += nt;
                    }
                }
        }
    }
}

/* ------------------------------------------------------------------ calibration sums (FP64) */
/* Unit-amplitude kernel f(x) of mass_update.cu:24-26 and -x f'(x), the per-pair quantities of
 * the calibration loss's evidence and of its length-scale derivative (x = d / ls). */
static double unit_f(double x) {
    double v = (2.0 + cos(M_PI * 2.0 * x)) * (1.0 - x) / 3.0 + sin(M_PI * 2.0 * x) / (2.0 * 3.141592);
    return v > 0.0 ? v : 0.0;
}
static double unit_mxfp(double x) {
    double v = (2.0 + cos(M_PI * 2.0 * x)) * (1.0 - x) / 3.0 + sin(M_PI * 2.0 * x) / (2.0 * 3.141592);
    if (!(v > 0.0)) return 0.0;
    double fp = (-2.0 * M_PI * sin(M_PI * 2.0 * x) * (1.0 - x) - (2.0 + cos(M_PI * 2.0 * x))) / 3.0 +
                2.0 * M_PI * cos(M_PI * 2.0 * x) / (2.0 * 3.141592);
    return -x * fp;
}

/* Distances of one (cell, point) pair as BGKI forms them (mass_update.cu:43-71): to the point
 * (occupied) and to the free segment when d_proj < d_m. */
static void pair_distances(double cx, double cy, double cz, double mx, double my, double mz, double res,
                           double* d_occ, double* d_free, int* has_free) {
    double dx = cx - mx, dy = cy - my, dz = cz - mz;
    *d_occ = sqrt(dx * dx + dy * dy + dz * dz);
    *has_free = 0;
    double dc = sqrt(cx * cx + cy * cy + cz * cz);
    double dm = sqrt(mx * mx + my * my + mz * mz);
    if (!(dm > 0.0)) return;
    double dp = (cx * mx + cy * my + cz * mz) / dm;
    double marg = fmax(0.9 * dm, dm - 2.0 * res);
    double df;
    if (dp <= 0.0) {
        df = dc;
    } else if (dp < marg) {
        double q = dc * dc - dp * dp;
        df = sqrt(q > 0.0 ? q : 0.0);
    } else {
        double r = marg / dm;
        double ex = cx - r * mx, ey = cy - r * my, ez = cz - r * mz;
        df = sqrt(ex * ex + ey * ey + ez * ez);
    }
    *d_free = df;
    *has_free = dp < dm;
}

/* Per cell: sum f(x) and sum -x f'(x) over the occupied pairs (Fo, Ho) and the free pairs
 * (Ff, Hf) within ls; enumeration as orc_bgki. */
void orc_bgki_sums(const orc_grid* g, double ls, int n, const float* xs, const float* ys, const float* zs,
                   double* Fo, double* Ff, double* Ho, double* Hf) {
    const int G = g->G, Gz = g->Gz;
    const int64_t C = (int64_t)G * G * Gz;
    memset(Fo, 0, sizeof(double) * C);
    memset(Ff, 0, sizeof(double) * C);
    memset(Ho, 0, sizeof(double) * C);
    memset(Hf, 0, sizeof(double) * C);
    const double res = g->res;
    const double R = ls / res + 1e-6;
    const double au[3] = {(double)g->sx / res + G / 2.0 - 0.5, (double)g->sy / res + G / 2.0 - 0.5,
                          (double)g->sz / res + Gz / 2.0 - 0.5};
    const int dims[3] = {G, G, Gz};
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
        const double m[3] = {xs[i], ys[i], zs[i]};
        if (!isfinite(m[0]) || !isfinite(m[1]) || !isfinite(m[2])) continue;
        const double bu[3] = {au[0] + m[0] / res, au[1] + m[1] / res, au[2] + m[2] / res};
        const double d[3] = {bu[0] - au[0], bu[1] - au[1], bu[2] - au[2]};
        int A = 0;
        if (fabs(d[1]) > fabs(d[A])) A = 1;
        if (fabs(d[2]) > fabs(d[A])) A = 2;
        const int Bx = (A + 1) % 3, Cx = (A + 2) % 3;
        int lo = (int)floor(fmin(au[A], bu[A]) - R), hi = (int)ceil(fmax(au[A], bu[A]) + R);
        if (lo < 0) lo = 0;
        if (hi > dims[A] - 1) hi = dims[A] - 1;
        for (int ia = lo; ia <= hi; ++ia) {
            double t0 = 0.0, t1 = 1.0;
            if (d[A] != 0.0) {
                double e0 = (ia - R - au[A]) / d[A], e1 = (ia + R - au[A]) / d[A];
                t0 = fmax(t0, fmin(e0, e1));
                t1 = fmin(t1, fmax(e0, e1));
                if (t0 > t1) continue;
            } else if (fabs(ia - au[A]) > R) {
                continue;
            }
            double b0 = au[Bx] + d[Bx] * t0, b1 = au[Bx] + d[Bx] * t1;
            double c0 = au[Cx] + d[Cx] * t0, c1 = au[Cx] + d[Cx] * t1;
            int ib0 = (int)floor(fmin(b0, b1) - R), ib1 = (int)ceil(fmax(b0, b1) + R);
            int ic0 = (int)floor(fmin(c0, c1) - R), ic1 = (int)ceil(fmax(c0, c1) + R);
            if (ib0 < 0) ib0 = 0;
            if (ic0 < 0) ic0 = 0;
            if (ib1 > dims[Bx] - 1) ib1 = dims[Bx] - 1;
            if (ic1 > dims[Cx] - 1) ic1 = dims[Cx] - 1;
            for (int ib = ib0; ib <= ib1; ++ib)
                for (int ic = ic0; ic <= ic1; ++ic) {
                    int idx3[3];
                    idx3[A] = ia;
                    idx3[Bx] = ib;
                    idx3[Cx] = ic;
                    float cxf, cyf, czf;
                    centre_f(g, idx3[0], idx3[1], idx3[2], &cxf, &cyf, &czf);
                    double dof, dfr;
                    int hf;
                    pair_distances(cxf, cyf, czf, m[0], m[1], m[2], res, &dof, &dfr, &hf);
                    const int occ_in = dof < ls, free_in = hf && dfr < ls;
                    if (!occ_in && !free_in) continue;
                    int64_t c = idx3[0] + (int64_t)G * idx3[1] + (int64_t)G * G * idx3[2];
                    if (occ_in) {
                        double x = dof / ls, a = unit_f(x), b = unit_mxfp(x);
#pragma omp atomic
                        Fo[c] += a;
#pragma omp atomic
                        Ho[c] += b;
                    }
                    if (free_in) {
                        double x = dfr / ls, a = unit_f(x), b = unit_mxfp(x);
#pragma omp atomic
                        Ff[c] += a;
#pragma omp atomic
                        Hf[c] += b;
                    }
                }
        }
    }
}

/* ------------------------------------------------------------------ K3DOM cell update (FP64) */
static double credit_d(double mass, double ms) { return 1.0 - 2.0 / (1.0 + exp(2.0 * mass / ms)); }
static double pdiff(double a, double b) { return a - b > 0.0 ? a - b : 0.0; }
static double ratio_d(double n, double r) { return (n <= 0.0 || r < 0.0) ? 0.0 : 1.0 / (1.0 + r / n); }

/* gridCellPredictionUpdateKernel (src/k3dom/kernel/mass_update.cu:152-183) with
 * predict_mass (:79-84), update_mass (:106-137), separate_newborn_part (:141-150), then the
 * per-cell parts of updatePersistentParticlesKernel2 (mu_UA) and statisticalMomentsKernel2
 * (mean velocity = mu_UA * sum(w v) / pers). has[c] = cell has particles (start != -1). */
void orc_k3dom_update(int C, double dt, double gamma, double p_B, double mass_scale, const double* del_occ,
                      const double* del_free, const float* free_in, const float* static_in, const float* dyn_in,
                      const int32_t* has, const double* sum_w, const double* swx, const double* swy,
                      const double* swz, double* o_free, double* o_static, double* o_dyn, double* o_born,
                      double* o_pers, double* o_pred, double* o_mu, double* o_mvx, double* o_mvy, double* o_mvz) {
    const double g = pow(gamma, dt);
#pragma omp parallel for schedule(static)
    for (int c = 0; c < C; ++c) {
        double mf = free_in[c], ms = static_in[c], md = dyn_in[c];
        double dp = has[c] ? sum_w[c] : 0.0;
        double pt = (mf + md) * g;
        ms *= g;
        md = fmin(dp, fmax(0.0, pt - ms));
        mf = pt - md;
        double dlf = del_free[c], dlo = del_occ[c];
        if (dlf > 0.0 || dlo > 0.0) {
            double ds = dlf + dlo, ps = mf + ms + md;
            double lD = 0, lS = 0, lF = 0;
            if (ps > 0.0) {
                double cr = credit_d(sqrt(ds * ps), mass_scale);
                lD = cr * pdiff(dlf, dlo) / ds * md / ps;
                lS = cr * pdiff(dlf, dlo) / ds * pdiff(ms + md, mf) / ps;
                lF = cr * pdiff(dlo, dlf) / ds * pdiff(mf, ms + md) / ps;
            }
            double df = lS / 2.0 * ms + lD * md - lF * mf;
            double dsm = -lS * ms;
            double dd = lF * mf + lS / 2.0 * ms - lD * md;
            mf += df;
            ms += dsm;
            md += dd;
            double cr2 = credit_d(ms + md, mass_scale);
            double beta = (1.0 - cr2) + cr2 * ratio_d(ms, md);
            ms = ms + beta * dlo;
            md = md + (1.0 - beta) * dlo;
            mf = mf + dlf;
        }
        double born;
        if (dp <= 0.0) born = md;
        else if (pt <= dp) born = 0.0;
        else born = (md * p_B * (pt - dp)) / (dp + p_B * (pt - dp));
        double pers = md - born;
        o_free[c] = mf;
        o_static[c] = ms;
        o_dyn[c] = md;
        o_born[c] = born;
        o_pers[c] = pers;
        o_pred[c] = dp;
        double mu = (has[c] && dp > 0.0) ? pers / dp : 0.0;
        o_mu[c] = mu;
        if (has[c] && pers > 0.0) {
            o_mvx[c] = mu * swx[c] / pers;
            o_mvy[c] = mu * swy[c] / pers;
            o_mvz[c] = mu * swz[c] / pers;
        } else {
            o_mvx[c] = o_mvy[c] = o_mvz[c] = 0.0;
        }
    }
}

/* ------------------------------------------------------------------ FP32 mirror of the reference */
/* The reference's own FP32 expressions (mass_update.cu:12-150), brute force over every
 * (cell, point) pair in input order, for pinning against the reference on small grids.
 * cospif/sinpif/expf/powf come from libm in double and are rounded to float (within an ulp
 * of CUDA's). nan_drop counts pairs whose radicand d_c^2 - d_proj^2 (:60) rounds negative in
 * FP32 -- sqrtf gives NaN and the reference silently drops a term that FP64 keeps. */
static float kernel_f(float d, float ls, float sigma) {
    float a = 2.0f * d;
    a = a / ls;
    float c = (float)cos(M_PI * (double)a), s = (float)sin(M_PI * (double)a);
    float t = 1.0f - d / ls;
    float v = (2.0f + c) * t;
    v = v / 3.0f;
    v = v + s / (2.0f * 3.141592f);
    v = sigma * v;
    return v > 0.0f ? v : 0.0f;
}

void orc_bgki_ref32(const orc_grid* g, float ls, float sigma, int n, const float* xs, const float* ys, const float* zs,
                    float* del_occ, float* del_free, int32_t* nan_drop) {
    const int G = g->G, Gz = g->Gz;
    const int64_t C = (int64_t)G * G * Gz;
    const float res = g->res;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t c = 0; c < C; ++c) {
        int ix = (int)(c % G), iy = (int)((c % ((int64_t)G * G)) / G), iz = (int)(c / ((int64_t)G * G));
        float x, y, z;
        centre_f(g, ix, iy, iz, &x, &y, &z);
        float occ = 0.0f, fr = 0.0f;
        int drops = 0;
        float dc = x * x;
        dc = dc + y * y;
        dc = dc + z * z;
        dc = sqrtf(dc);
        for (int i = 0; i < n; ++i) {
            float xm = xs[i], ym = ys[i], zm = zs[i];
            float a = (x - xm) * (x - xm);
            a = a + (y - ym) * (y - ym);
            a = a + (z - zm) * (z - zm);
            float d = sqrtf(a);
            if (d < ls) occ += kernel_f(d, ls, sigma);
            float dm = xm * xm;
            dm = dm + ym * ym;
            dm = dm + zm * zm;
            dm = sqrtf(dm);
            float dp = x * xm;
            dp = dp + y * ym;
            dp = dp + z * zm;
            dp = dp / dm;
            float marg = fmaxf(0.9f * dm, dm - 2.0f * res);
            if (dp <= 0.0f) {
                d = dc;
            } else if (dp < marg) {
                float q = dc * dc - dp * dp;
                if (q < 0.0f) drops++;
                d = sqrtf(q);
            } else if (dp < dm) {
                float r = marg / dm;
                float ex = (x - r * xm) * (x - r * xm);
                ex = ex + (y - r * ym) * (y - r * ym);
                ex = ex + (z - r * zm) * (z - r * zm);
                d = sqrtf(ex);
            } else {
                d = ls + 1.0f;
            }
            if (d < ls) fr += kernel_f(d, ls, sigma);
        }
        del_occ[c] = occ;
        del_free[c] = fr;
        nan_drop[c] = drops;
    }
}

/* gridCellPredictionUpdateKernel's per-cell body in FP32 (mass_update.cu:79-150, 163-181). */
void orc_k3dom_update_ref32(int C, float dt, float gamma, float p_B, float mass_scale, const float* del_occ,
                            const float* del_free, const float* free_in, const float* static_in, const float* dyn_in,
                            const float* dyn_pred, float* o_free, float* o_static, float* o_dyn, float* o_born,
                            float* o_pers) {
    const float g = (float)pow((double)gamma, (double)dt);
    for (int c = 0; c < C; ++c) {
        float mf = free_in[c], ms = static_in[c], md = dyn_in[c], dp = dyn_pred[c];
        float pt = (mf + md) * g;
        ms = ms * g;
        md = fminf(dp, fmaxf(0.0f, pt - ms));
        mf = pt - md;
        float dlf = del_free[c], dlo = del_occ[c];
        if (dlf > 0.0f || dlo > 0.0f) {
            float ds = dlf + dlo;
            float ps = mf + ms;
            ps = ps + md;
            float cr = 1.0f - 2.0f / (1.0f + (float)exp((double)(2.0f * sqrtf(ds * ps) / mass_scale)));
            float pdf = fmaxf(0.0f, dlf - dlo), pdo = fmaxf(0.0f, dlo - dlf);
            float lD = cr * pdf;
            lD = lD / ds;
            lD = lD * md;
            lD = lD / ps;
            float lS = cr * pdf;
            lS = lS / ds;
            lS = lS * fmaxf(0.0f, (ms + md) - mf);
            lS = lS / ps;
            float lF = cr * pdo;
            lF = lF / ds;
            lF = lF * fmaxf(0.0f, mf - (ms + md));
            lF = lF / ps;
            float df = (lS / 2.0f) * ms;
            df = df + lD * md;
            df = df - lF * mf;
            float dsm = -lS * ms;
            float dd = lF * mf;
            dd = dd + (lS / 2.0f) * ms;
            dd = dd - lD * md;
            mf = mf + df;
            ms = ms + dsm;
            md = md + dd;
            float cr2 = 1.0f - 2.0f / (1.0f + (float)exp((double)(2.0f * (ms + md) / mass_scale)));
            float ratio = (ms <= 0.0f || md < 0.0f) ? 0.0f : 1.0f / (1.0f + md / ms);
            float beta = (1.0f - cr2) + cr2 * ratio;
            ms = ms + beta * dlo;
            md = md + (1.0f - beta) * dlo;
            mf = mf + dlf;
        }
        float born;
        if (dp <= 0.0f) born = md;
        else if (pt <= dp) born = 0.0f;
        else {
            float a = md * p_B;
            a = a * (pt - dp);
            float b = p_B * (pt - dp);
            b = dp + b;
            born = a / b;
        }
        o_free[c] = mf;
        o_static[c] = ms;
        o_dyn[c] = md;
        o_born[c] = born;
        o_pers[c] = md - born;
    }
}

/* ------------------------------------------------------------------ DS-PHD/MIB */
/* Neighbour test of calcMeasurementGridKernel (measurement_grid.cu:88-99), FP32 order. */
static int ds_nbr(float x, float y, float z, float acs, float mx, float my, float mz, float ams, float wr2) {
    float ip = x * mx;
    ip = ip + y * my;
    ip = ip + z * mz;
    float q = ip * ip;
    q = q / ams;
    return ip > 0.0f && (acs - q) < wr2;
}

/* Measurement grid (measurement_grid.cu:64-162): per cell the first <= 100 rays, in input
 * order, whose line passes within the window; then the inverse sensor model. The neighbour
 * set is decided in FP32 exactly as the reference; pOcc uses libm expf, so the two
 * comparisons on it (:123, :136) are reported in tie[] when within 4 ulp of flipping.
 * Rays are binned to 8x8x8-cell blocks first (conservative), keeping input order. */
void orc_ds_measgrid(const orc_grid* g, float max_range, float delta, int n, const float* xs, const float* ys,
                     const float* zs, float* meas_occ, float* meas_free, int32_t* nbr_count, int32_t* tie) {
    const int G = g->G, Gz = g->Gz;
    const float res = g->res;
    const float wr = res * 0.866f;
    const float wr2 = wr * wr;
    const int BS = 8;
    const int nbx = (G + BS - 1) / BS, nbz = (Gz + BS - 1) / BS;
    const int64_t NB = (int64_t)nbx * nbx * nbz;
    /* conservative radius (cells) */
    double ext = 2.0 * ((double)G * res * 1.7320508 + (double)Gz * res);
    double Rm = sqrt((double)wr2 + 64.0 * 5.96e-8 * ext * ext) + 1e-3 * res;
    double R = Rm / res + 0.87 * BS; /* block half diagonal slack handled by testing block boxes */
    (void)R;
    int64_t* cnt = (int64_t*)calloc((size_t)NB + 1, sizeof(int64_t));
    const double au[3] = {(double)g->sx / res + G / 2.0 - 0.5, (double)g->sy / res + G / 2.0 - 0.5,
                          (double)g->sz / res + Gz / 2.0 - 0.5};
    const double Rc = Rm / res;
    /* pass 1 count, pass 2 fill (ray order preserved per block) */
    int64_t* off = NULL;
    int32_t* lists = NULL;
    for (int pass = 0; pass < 2; ++pass) {
        int64_t* cur = NULL;
        if (pass == 1) {
            off = (int64_t*)calloc((size_t)NB + 1, sizeof(int64_t));
            for (int64_t b = 0; b < NB; ++b) off[b + 1] = off[b] + cnt[b];
            lists = (int32_t*)malloc(sizeof(int32_t) * (size_t)(off[NB] + 1));
            cur = (int64_t*)malloc(sizeof(int64_t) * (size_t)NB);
            memcpy(cur, off, sizeof(int64_t) * (size_t)NB);
        }
        for (int i = 0; i < n; ++i) {
            double m[3] = {xs[i], ys[i], zs[i]};
            double len = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
            if (!(len > 0.0) || !isfinite(len)) continue;
            double u[3] = {m[0] / len, m[1] / len, m[2] / len};
            for (int bz = 0; bz < nbz; ++bz)
                for (int by = 0; by < nbx; ++by)
                    for (int bx = 0; bx < nbx; ++bx) {
                        /* distance from the block's centre-box to the half-line, conservative */
                        double lo[3] = {bx * BS - Rc, by * BS - Rc, bz * BS - Rc};
                        double hi[3] = {bx * BS + BS - 1 + Rc, by * BS + BS - 1 + Rc, bz * BS + BS - 1 + Rc};
                        double t0 = 0.0, t1 = 1e30;
                        int ok = 1;
                        for (int k = 0; k < 3 && ok; ++k) {
                            if (u[k] == 0.0) {
                                if (au[k] < lo[k] || au[k] > hi[k]) ok = 0;
                            } else {
                                double e0 = (lo[k] - au[k]) / u[k], e1 = (hi[k] - au[k]) / u[k];
                                t0 = fmax(t0, fmin(e0, e1));
                                t1 = fmin(t1, fmax(e0, e1));
                                if (t0 > t1) ok = 0;
                            }
                        }
                        if (!ok) continue;
                        int64_t b = bx + (int64_t)nbx * (by + (int64_t)nbx * bz);
                        if (pass == 0) cnt[b]++;
                        else lists[cur[b]++] = i;
                    }
        }
        if (pass == 1) free(cur);
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t b = 0; b < NB; ++b) {
        int bx = (int)(b % nbx), by = (int)((b / nbx) % nbx), bz = (int)(b / ((int64_t)nbx * nbx));
        for (int lz = 0; lz < BS; ++lz)
            for (int ly = 0; ly < BS; ++ly)
                for (int lx = 0; lx < BS; ++lx) {
                    int ix = bx * BS + lx, iy = by * BS + ly, iz = bz * BS + lz;
                    if (ix >= G || iy >= G || iz >= Gz) continue;
                    int64_t c = ix + (int64_t)G * iy + (int64_t)G * G * iz;
                    float x, y, z;
                    centre_f(g, ix, iy, iz, &x, &y, &z);
                    float acs = x * x;
                    acs = acs + y * y;
                    acs = acs + z * z;
                    int nb = 0, all_far = 1, tie_c = 0;
                    float mx = 0.0f;
                    for (int64_t e = off[b]; e < off[b + 1] && nb < 100; ++e) {
                        int i = lists[e];
                        float ax = xs[i], ay = ys[i], az = zs[i];
                        float ams = ax * ax;
                        ams = ams + ay * ay;
                        ams = ams + az * az;
                        if (!ds_nbr(x, y, z, acs, ax, ay, az, ams, wr2)) continue;
                        nb++;
                        if (acs > ams) all_far = 0;
                        float dx = x - ax, dy = y - ay, dz = z - az;
                        float rs = dx * dx;
                        rs = rs + dy * dy;
                        rs = rs + dz * dz;
                        float ds2 = delta * delta;
                        float o = 0.95f * expf((-0.5f * rs) / ds2);
                        if (o > mx) mx = o;
                    }
                    float mo, mf;
                    if (nb == 0) {
                        mo = mf = 0.0f;
                    } else {
                        if (all_far) {
                            float r = sqrtf(acs);
                            float unc = r / max_range;
                            unc = unc * (1.0f - 0.15f);
                            unc = 0.15f + unc;
                            if (fabsf(mx - unc) <= 4.0f * FLT_EPSILON * fmaxf(mx, unc)) tie_c = 1;
                            if (mx > unc) {
                                mo = mx;
                                mf = 0.0f;
                            } else {
                                mo = 0.0f;
                                mf = 1.0f - unc;
                            }
                        } else {
                            if (fabsf(mx - 0.5f) <= 4.0f * FLT_EPSILON) tie_c = 1;
                            mo = mx > 0.5f ? mx : 0.0f;
                            mf = 0.0f;
                        }
                        const float eps = 0.00001f;
                        mo = fmaxf(eps, fminf(1.0f - eps, mo));
                        mf = fmaxf(eps, fminf(1.0f - eps, mf));
                    }
                    meas_occ[c] = mo;
                    meas_free[c] = mf;
                    nbr_count[c] = nb;
                    tie[c] = tie_c;
                }
    }
    free(cnt);
    free(off);
    free(lists);
}

/* DS gridCellPredictionUpdateKernel (src/dsphdmib/kernel/mass_update.cu:46-87) in FP64:
 * in-place normalisation (w /= occ_pred when > 1) is reported through o_div, Dempster
 * combination (:17-30), birth split (:32-35), then mu_UA and the mean velocity. */
void orc_ds_update(int C, double p_B, const float* meas_occ, const float* meas_free, const float* occ_in,
                   const float* free_in, const int32_t* has, const double* sum_w, const double* swx,
                   const double* swy, const double* swz, double* o_occ, double* o_free, double* o_born,
                   double* o_pers, double* o_pred, double* o_mu, double* o_div, double* o_mvx, double* o_mvy,
                   double* o_mvz) {
#pragma omp parallel for schedule(static)
    for (int c = 0; c < C; ++c) {
        double mo = meas_occ[c], mfm = meas_free[c];
        double op, fp, born = 0.0, pred = 0.0, div = 0.0;
        if (has[c]) {
            op = sum_w[c];
            if (op > 1.0) {
                div = op;
                op = 1.0;
            }
            fp = fmin(0.9 * (double)free_in[c], 1.0 - op);
            pred = op;
        } else {
            op = occ_in[c];
            fp = fmin(0.9 * (double)free_in[c], 1.0 - op);
        }
        double up = 1.0 - op - fp, mu_ = 1.0 - mfm - mo, K = fp * mo + op * mfm;
        double occ = (op * mu_ + up * mo + op * mo) / (1.0 - K);
        double fr = (fp * mu_ + up * mfm + fp * mfm) / (1.0 - K);
        if (has[c]) born = (occ * p_B * (1.0 - op)) / (op + p_B * (1.0 - op));
        double pers = occ - born;
        o_occ[c] = occ;
        o_free[c] = fr;
        o_born[c] = born;
        o_pers[c] = pers;
        o_pred[c] = pred;
        o_div[c] = div;
        double mu = (has[c] && pred > 0.0) ? pers / pred : 0.0;
        o_mu[c] = mu;
        double s = div > 0.0 ? div : 1.0;
        if (has[c] && pers > 0.0) {
            o_mvx[c] = mu * swx[c] / s / pers;
            o_mvy[c] = mu * swy[c] / s / pers;
            o_mvz[c] = mu * swz[c] / s / pers;
        } else {
            o_mvx[c] = o_mvy[c] = o_mvz[c] = 0.0;
        }
    }
}

/* ------------------------------------------------------------------ exact scans */
static u128 to_fixed(float f) {
    uint32_t b;
    memcpy(&b, &f, 4);
    if (b & 0x80000000u) return 0;
    uint32_t e = b >> 23, frac = b & 0x7FFFFFu;
    if (e == 0xFFu) return 0;
    uint32_t m = e ? (frac | 0x800000u) : frac;
    int sh = (e ? (int)e : 1) - 150 + 80;
    if (sh >= 0) {
        if (sh > 127 - 24) return 0;
        return (u128)m << sh;
    }
    if (sh <= -32) return 0;
    return (u128)(m >> (-sh));
}
static float from_fixed(u128 v) { return ldexpf((float)v, -80); }

/* Inclusive prefix sums of a[0..na) ++ b[0..nb), exact and rounded once to float. */
void orc_exact_scan(int64_t na, const float* a, int64_t nb, const float* b, float* out) {
    u128 s = 0;
    for (int64_t i = 0; i < na; ++i) {
        s += to_fixed(a[i]);
        out[i] = from_fixed(s);
    }
    for (int64_t i = 0; i < nb; ++i) {
        s += to_fixed(b[i]);
        out[na + i] = from_fixed(s);
    }
}

/* ------------------------------------------------------------------ births and first frame */
/* Slot ranges (init_new_particles.cu:14-27, normalize_particle_orders :44-52):
 * bound(j) = int(cum[j] * (v / cum[C-1])); cell j owns [bound(j-1), bound(j) - 1]. */
static int owner_of(const float* cum, int C, float k, int s) {
    int lo = 0, hi = C;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (f2i(cum[mid] * k) > s) hi = mid; else lo = mid + 1;
    }
    return lo;
}

static void vel_draw(float u0, float u1, float u2, float vmax, float min_vel, float* o) {
    float lo = -vmax, hi = vmax, span = hi - lo;
    float x = span * (1.0f - u0), y = span * (1.0f - u1), z = span * (1.0f - u2);
    x = lo + x;
    y = lo + y;
    z = lo + z;
    float vsq = x * x;
    vsq = vsq + y * y;
    vsq = vsq + z * z;
    if (vsq < min_vel * min_vel && vsq != 0.0f) {
        float rate = min_vel / sqrtf(vsq);
        x = x * rate;
        y = y * rate;
        z = z * rate;
    }
    o[0] = x;
    o[1] = y;
    o[2] = z;
}

/* initNewParticlesKernel1/2 (init_new_particles.cu:106-183). cum = exact prefix of born.
 * Slots past the last cell's range keep (cell, assoc) from before, as in the reference.
 * out_w is the weight before the resampling penalty; slow[] marks the penalty
 * (resampling.cu:35-42). uniforms: 3 per slot (stage 3). */
void orc_births(int C, int B, int G, float p_A, float vmax, float min_vel, const float* born, const float* cum,
                const float* uniforms, int32_t* cell, uint8_t* assoc, float* pos, float* vel, float* w,
                uint8_t* slow) {
    float k = (float)B / cum[C - 1];
    for (int s = 0; s < B; ++s) {
        int j = owner_of(cum, C, k, s);
        int n, st;
        int as;
        if (j < C) {
            st = j == 0 ? 0 : f2i(cum[j - 1] * k);
            n = f2i(cum[j] * k) - st;
            int nuA0 = (int)roundf((float)n * p_A);
            as = s < st + nuA0;
            cell[s] = j;
            assoc[s] = (uint8_t)as;
        } else {
            j = clampi(cell[s], 0, C - 1);
            as = assoc[s] != 0;
            int b1 = f2i(cum[j] * k), b0 = j == 0 ? 0 : f2i(cum[j - 1] * k);
            n = b0 <= b1 - 1 ? b1 - b0 : 0;
        }
        int nuA = (int)roundf((float)n * p_A), nuUA = n - nuA;
        float bm = born[j];
        float ww;
        if (as) ww = nuA > 0 ? (p_A * bm) / (float)nuA : 0.0f;
        else ww = nuUA > 0 ? (float)((1.0 - (double)p_A) * (double)bm / (double)nuUA) : 0.0f;
        int ix = j % G, iy = (j % (G * G)) / G, iz = j / (G * G);
        pos[3 * s] = (float)ix + 0.5f;
        pos[3 * s + 1] = (float)iy + 0.5f;
        pos[3 * s + 2] = (float)iz + 0.5f;
        vel_draw(uniforms[3 * s], uniforms[3 * s + 1], uniforms[3 * s + 2], vmax, min_vel, vel + 3 * s);
        float sp = vel[3 * s] * vel[3 * s];
        sp = sp + vel[3 * s + 1] * vel[3 * s + 1];
        sp = sp + vel[3 * s + 2] * vel[3 * s + 2];
        slow[s] = sp < min_vel * min_vel;
        w[s] = ww;
    }
}

/* initParticlesKernel1/2 (init_new_particles.cu:54-104): first frame, v = P. */
void orc_init_particles(int C, int P, int G, float vmax, float min_vel, const float* cum, const float* uniforms,
                        int32_t* cell, float* pos, float* vel, float* w) {
    float k = (float)P / cum[C - 1];
    for (int s = 0; s < P; ++s) {
        int j = owner_of(cum, C, k, s);
        if (j < C) cell[s] = j;
        else j = clampi(cell[s], 0, C - 1);
        int ix = j % G, iy = (j % (G * G)) / G, iz = j / (G * G);
        pos[3 * s] = (float)ix + 0.5f;
        pos[3 * s + 1] = (float)iy + 0.5f;
        pos[3 * s + 2] = (float)iz + 0.5f;
        vel_draw(uniforms[3 * s], uniforms[3 * s + 1], uniforms[3 * s + 2], vmax, min_vel, vel + 3 * s);
        w[s] = 1.0f / (float)P;
    }
}

/* ------------------------------------------------------------------ resampling */
static int cmp_u32(const void* a, const void* b) {
    uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
    return (x > y) - (x < y);
}

/* resampling() (src/common/dom.cu:259-297; resampling.cu:13-89): joint = sorted persistent
 * weights ++ birth weights (penalties already applied), exact prefix, draws
 * u = joint_max * (1 - U) sorted ascending, the last prefix replaced by the largest draw,
 * ancestor = lower_bound. Returns joint_max; writes the ancestors and the exact prefix. */
float orc_resample(int P, int B, const float* w_sorted, const float* w_birth, uint64_t seed, uint32_t frame,
                   int32_t* anc, float* cum) {
    const int64_t n = (int64_t)P + B;
    orc_exact_scan(P, w_sorted, B, w_birth, cum);
    const float jmax = cum[n - 1];
    uint32_t* keys = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)P);
    orc_resample_keys(seed, frame, P, keys);
    qsort(keys, (size_t)P, sizeof(uint32_t), cmp_u32);
    const float rmax = (jmax * ((float)keys[P - 1] * 5.9604644775390625e-08f)) + 0.0f;
    const float last = cum[n - 1];
    cum[n - 1] = rmax; /* calc_resampled_indices (:58-63) */
    int64_t j = 0;
    for (int k = 0; k < P; ++k) {
        float u = (jmax * ((float)keys[k] * 5.9604644775390625e-08f)) + 0.0f;
        while (j < n && cum[j] < u) ++j;
        anc[k] = (int32_t)(j < n ? j : n - 1);
    }
    cum[n - 1] = last;
    free(keys);
    return jmax;
}

/* Resampling from a given cumulative array and sorted draws, the integer rule alone:
 * lower_bound with the last element replaced by the largest draw when they differ. */
void orc_lower_bound_rule(int64_t n, const float* cum_in, int64_t P, const float* sorted_u, int32_t* anc) {
    float* cum = (float*)malloc(sizeof(float) * (size_t)n);
    memcpy(cum, cum_in, sizeof(float) * (size_t)n);
    if (cum[n - 1] != sorted_u[P - 1]) cum[n - 1] = sorted_u[P - 1];
    for (int64_t k = 0; k < P; ++k) {
        int64_t lo = 0, hi = n;
        while (lo < hi) {
            int64_t mid = (lo + hi) >> 1;
            if (cum[mid] < sorted_u[k]) lo = mid + 1; else hi = mid;
        }
        anc[k] = (int32_t)lo;
    }
    free(cum);
}

/* Birth slot boundaries from a given cumulative array (the integer rule alone). */
void orc_slot_bounds(int C, const float* cum, int v, int32_t* start, int32_t* end) {
    float k = (float)v / cum[C - 1];
    for (int j = 0; j < C; ++j) {
        start[j] = j == 0 ? 0 : f2i(cum[j - 1] * k);
        end[j] = f2i(cum[j] * k) - 1;
    }
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
