/*
 * k3dom_calib_oracle.c -- TEST INFRASTRUCTURE ONLY. The FP64 reference of the differentiable
 * kernel-inference update: the calibration loss and its gradient by forward-mode dual numbers
 * (an implementation independent of the library's hand-written reverse-mode adjoint), and the
 * held-out labels by 3-D DDA.
 *
 * Model (per cell; masses in FP64, the K3DOM cell update of src/k3dom/kernel/mass_update.cu:79-139):
 *   theta = (ls, sigma, gamma, occupied prior, free prior); E = sigma * sum f(d / ls), where the
 *   per-cell sums F (of f) and H (of -x f'(x), so dE/dls = sigma H / ls) come from
 *   orc_bgki_sums. Frame 0 starts from the priors (free = theta_free, static = dynamic =
 *   theta_occ / 2) with dt = 0 and no particles; frame k predicts with gamma^dt_k and the given
 *   particle weight sum dyn_k(c), then updates with E_k. p = (static + dynamic) / total.
 *   Loss = sum_c (-n1 log p - n0 log(1 - p)) / (sum n0 + n1), p clamped to [1e-7, 1 - 1e-7].
 * Compiled with -ffp-contract=off.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ND 5 /* ls, sigma, gamma, prior_occ, prior_free */

typedef struct {
    double v;
    double d[ND];
} dual;

static dual dc(double v) {
    dual r;
    r.v = v;
    memset(r.d, 0, sizeof(r.d));
    return r;
}
static dual dadd(dual a, dual b) {
    dual r;
    r.v = a.v + b.v;
    for (int i = 0; i < ND; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
static dual dsub(dual a, dual b) {
    dual r;
    r.v = a.v - b.v;
    for (int i = 0; i < ND; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
static dual dmul(dual a, dual b) {
    dual r;
    r.v = a.v * b.v;
    for (int i = 0; i < ND; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
static dual ddiv(dual a, dual b) {
    dual r;
    r.v = a.v / b.v;
    for (int i = 0; i < ND; ++i) r.d[i] = (a.d[i] * b.v - a.v * b.d[i]) / (b.v * b.v);
    return r;
}
static dual dscale(dual a, double s) {
    dual r;
    r.v = a.v * s;
    for (int i = 0; i < ND; ++i) r.d[i] = a.d[i] * s;
    return r;
}
static dual dsqrt(dual a) {
    dual r;
    r.v = sqrt(a.v);
    for (int i = 0; i < ND; ++i) r.d[i] = r.v > 0.0 ? a.d[i] / (2.0 * r.v) : 0.0;
    return r;
}
static dual dexp(dual a) {
    dual r;
    r.v = exp(a.v);
    for (int i = 0; i < ND; ++i) r.d[i] = a.d[i] * r.v;
    return r;
}
static dual dlog(dual a) {
    dual r;
    r.v = log(a.v);
    for (int i = 0; i < ND; ++i) r.d[i] = a.d[i] / a.v;
    return r;
}
/* the branch of the value decides which operand (and derivative) is taken */
static dual dmax(dual a, dual b) { return a.v >= b.v ? a : b; }
static dual dmin(dual a, dual b) { return a.v <= b.v ? a : b; }

static dual credit(dual x, double ms) {
    /* value 1 - 2 / (1 + exp(2 x / ms)) (mass_update.cu:12-14); derivative (4 / ms) t / (1 + t)^2
     * with t = exp(-|2 x / ms|), which stays finite where exp(2 x / ms) overflows */
    dual r;
    r.v = 1.0 - 2.0 / (1.0 + exp(2.0 * x.v / ms));
    const double t = exp(-fabs(2.0 * x.v / ms));
    const double dv = (4.0 / ms) * t / ((1.0 + t) * (1.0 + t));
    for (int i = 0; i < ND; ++i) r.d[i] = x.d[i] * dv;
    return r;
}

static void frame_update(dual* mf, dual* ms, dual* md, dual g, double dyn, dual Eo, dual Ef, double mass_scale) {
    dual P = dmul(dadd(*mf, *md), g);
    dual s1 = dmul(*ms, g);
    dual d1 = dmin(dc(dyn), dmax(dc(0.0), dsub(P, s1)));
    dual f1 = dsub(P, d1);
    if (!(Ef.v > 0.0 || Eo.v > 0.0)) {
        *mf = f1;
        *ms = s1;
        *md = d1;
        return;
    }
    dual Sd = dadd(Ef, Eo);
    dual Sp = dadd(dadd(f1, s1), d1);
    dual lDF = dc(0.0), lSFD = dc(0.0), lFD = dc(0.0);
    if (Sp.v > 0.0) {
        dual cr = credit(dsqrt(dmul(Sd, Sp)), mass_scale);
        dual bf = ddiv(dmul(cr, dmax(dc(0.0), dsub(Ef, Eo))), Sd);
        dual bo = ddiv(dmul(cr, dmax(dc(0.0), dsub(Eo, Ef))), Sd);
        lDF = ddiv(dmul(bf, d1), Sp);
        lSFD = ddiv(dmul(bf, dmax(dc(0.0), dsub(dadd(s1, d1), f1))), Sp);
        lFD = ddiv(dmul(bo, dmax(dc(0.0), dsub(f1, dadd(s1, d1)))), Sp);
    }
    dual f2 = dsub(dadd(dadd(f1, dmul(dscale(lSFD, 0.5), s1)), dmul(lDF, d1)), dmul(lFD, f1));
    dual s2 = dsub(s1, dmul(lSFD, s1));
    dual d2 = dsub(dadd(dadd(d1, dmul(lFD, f1)), dmul(dscale(lSFD, 0.5), s1)), dmul(lDF, d1));
    dual cr2 = credit(dadd(s2, d2), mass_scale);
    dual r = (s2.v <= 0.0 || d2.v < 0.0) ? dc(0.0) : ddiv(dc(1.0), dadd(dc(1.0), ddiv(d2, s2)));
    dual beta = dadd(dsub(dc(1.0), cr2), dmul(cr2, r));
    *ms = dadd(s2, dmul(beta, Eo));
    *md = dadd(d2, dmul(dsub(dc(1.0), beta), Eo));
    *mf = dadd(f2, Ef);
}

/* sums: F frames x 4 x C (f occ, f free, -x f' occ, -x f' free) evaluated at theta[0];
 * dyn: F x C (frame 0 ignored; NULL rows allowed via dyn_present[k] == 0). Returns the loss;
 * grad (may be NULL) receives dLoss/dtheta. */
double orc_calib_loss_grad(int64_t C, int F, const double* sums, const float* dt, const float* dyn,
                           const int32_t* dyn_present, const uint32_t* n0, const uint32_t* n1,
                           const double* theta, double mass_scale, double* grad) {
    double total = 0.0;
    for (int64_t c = 0; c < C; ++c) total += (double)n0[c] + (double)n1[c];
    if (!(total > 0.0)) {
        if (grad) memset(grad, 0, sizeof(double) * ND);
        return 0.0;
    }
    double loss = 0.0;
    double g[ND] = {0, 0, 0, 0, 0};
#pragma omp parallel
    {
        double loss_l = 0.0, g_l[ND] = {0, 0, 0, 0, 0};
#pragma omp for schedule(static)
        for (int64_t c = 0; c < C; ++c) {
            if (n0[c] == 0 && n1[c] == 0) continue;
            /* ls enters through dE/dls below; gamma through g_k */
            dual sigma = dc(theta[1]);
            sigma.d[1] = 1.0;
            dual po = dc(theta[3]), pf = dc(theta[4]);
            po.d[3] = 1.0;
            pf.d[4] = 1.0;
            dual mf = pf, ms = dscale(po, 0.5), md = dscale(po, 0.5);
            for (int k = 0; k < F; ++k) {
                const double* s = sums + (int64_t)k * 4 * C;
                /* E = sigma F with dE/dls = sigma H / ls */
                dual Eo = dscale(sigma, s[c]), Ef = dscale(sigma, s[C + c]);
                Eo.d[0] = theta[1] * s[2 * C + c] / theta[0];
                Ef.d[0] = theta[1] * s[3 * C + c] / theta[0];
                dual gk;
                if (k == 0) {
                    gk = dc(1.0);
                } else {
                    gk = dc(pow(theta[2], (double)dt[k]));
                    gk.d[2] = (double)dt[k] * pow(theta[2], (double)dt[k] - 1.0);
                }
                double dynv = (k > 0 && dyn_present[k]) ? (double)dyn[(int64_t)k * C + c] : 0.0;
                frame_update(&mf, &ms, &md, gk, dynv, Eo, Ef, mass_scale);
            }
            dual T = dadd(dadd(mf, ms), md);
            dual p = ddiv(dadd(ms, md), T);
            const double lo = 1e-7, hi = 1.0 - 1e-7;
            if (p.v < lo) p = dc(lo);
            if (p.v > hi) p = dc(hi);
            dual l = dsub(dscale(dlog(p), -(double)n1[c]), dscale(dlog(dsub(dc(1.0), p)), (double)n0[c]));
            loss_l += l.v;
            for (int i = 0; i < ND; ++i) g_l[i] += l.d[i];
        }
#pragma omp critical
        {
            loss += loss_l;
            for (int i = 0; i < ND; ++i) g[i] += g_l[i];
        }
    }
    if (grad)
        for (int i = 0; i < ND; ++i) grad[i] = g[i] / total;
    return loss / total;
}

/* Occupancy p(c) after the frames at theta (values only). */
void orc_calib_occupancy(int64_t C, int F, const double* sums, const float* dt, const float* dyn,
                         const int32_t* dyn_present, const double* theta, double mass_scale, double* p_out) {
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < C; ++c) {
        dual mf = dc(theta[4]), ms = dc(theta[3] * 0.5), md = dc(theta[3] * 0.5);
        for (int k = 0; k < F; ++k) {
            const double* s = sums + (int64_t)k * 4 * C;
            dual Eo = dc(theta[1] * s[c]), Ef = dc(theta[1] * s[C + c]);
            dual gk = dc(k == 0 ? 1.0 : pow(theta[2], (double)dt[k]));
            double dynv = (k > 0 && dyn_present[k]) ? (double)dyn[(int64_t)k * C + c] : 0.0;
            frame_update(&mf, &ms, &md, gk, dynv, Eo, Ef, mass_scale);
        }
        double T = mf.v + ms.v + md.v;
        p_out[c] = T > 0.0 ? (ms.v + md.v) / T : 0.5;
    }
}

/* Held-out labels: Amanatides-Woo traversal in continuous index space X = x / res + G / 2 from
 * the sensor s to the hit s + m; voxels before the hit voxel count n0, the hit voxel n1;
 * voxels outside the grid are skipped; ties x before y before z. */
void orc_dda_labels(int G, int Gz, double res, float sx, float sy, float sz, int n, const float* xyz, uint32_t* n0,
                    uint32_t* n1) {
    const double half[3] = {G / 2.0, G / 2.0, Gz / 2.0};
    const int dims[3] = {G, G, Gz};
    for (int i = 0; i < n; ++i) {
        const double m[3] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
        if (!isfinite(m[0]) || !isfinite(m[1]) || !isfinite(m[2])) continue;
        const double s[3] = {sx, sy, sz};
        double a[3], b[3], tmax[3], tdel[3];
        int v[3], e[3], step[3];
        long budget = 1;
        for (int k = 0; k < 3; ++k) {
            a[k] = s[k] / res + half[k];
            b[k] = (s[k] + m[k]) / res + half[k];
            v[k] = (int)floor(a[k]);
            e[k] = (int)floor(b[k]);
            const double d = b[k] - a[k];
            budget += labs((long)e[k] - v[k]);
            if (d > 0.0) {
                step[k] = 1;
                tdel[k] = 1.0 / d;
                tmax[k] = ((double)(v[k] + 1) - a[k]) * tdel[k];
            } else if (d < 0.0) {
                step[k] = -1;
                tdel[k] = -1.0 / d;
                tmax[k] = (a[k] - (double)v[k]) * tdel[k];
            } else {
                step[k] = 0;
                tdel[k] = INFINITY;
                tmax[k] = INFINITY;
            }
        }
        for (long it = 0; it < budget; ++it) {
            if (v[0] == e[0] && v[1] == e[1] && v[2] == e[2]) break;
            if (v[0] >= 0 && v[0] < dims[0] && v[1] >= 0 && v[1] < dims[1] && v[2] >= 0 && v[2] < dims[2])
                n0[v[0] + (int64_t)G * v[1] + (int64_t)G * G * v[2]] += 1;
            int k = 0;
            if (tmax[1] < tmax[k]) k = 1;
            if (tmax[2] < tmax[k]) k = 2;
            v[k] += step[k];
            tmax[k] = tmax[k] + tdel[k];
        }
        if (e[0] >= 0 && e[0] < dims[0] && e[1] >= 0 && e[1] < dims[1] && e[2] >= 0 && e[2] < dims[2])
            n1[e[0] + (int64_t)G * e[1] + (int64_t)G * G * e[2]] += 1;
    }
}
