/*
 * ORACLE -- test infrastructure, not product code.
 *
 * A plain, single-threaded C restatement of the reference's per-turn
 * particle routines.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load this library, and only to check (never to produce)
 * results of the CUDA engine.  Every function names the reference routine it
 * restates.  It is compiled WITHOUT fast-math and WITHOUT FP contraction so
 * its rounding is the plain IEEE sequence of the source expressions.
 *
 * Parity pins: tests/test_oracle_golden.py checks this library against the
 * reference's own golden vectors (unittests/beam_profile/
 * test_beam_profile_object.py:169-230) and against the reference's compiled
 * C++ (oracle/_ref) on seeded inputs.
 *
 * Each routine exists for double (suffix _f64) and float (_f32), mirroring
 * libblond_double.so / libblond_single.so (blond_common.h:22-36).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

#define DEFINE_ORACLE(real, SUF, SIN, FLOOR, SQRT)                              \
                                                                              \
/* kick.cpp:16-35: dE += charge * sum_j V_j sin(omega_j dt + phi_j) + acc */  \
void oracle_kick_##SUF(const real *dt, real *dE, int n_rf, real charge,       \
                       const real *voltage, const real *omega_rf,             \
                       const real *phi_rf, int n, real acc_kick)              \
{                                                                             \
    for (int i = 0; i < n; ++i) {                                             \
        real s = 0;                                                           \
        const real t = dt[i];                                                 \
        for (int j = 0; j < n_rf; ++j)                                        \
            s += voltage[j] * SIN(omega_rf[j] * t + phi_rf[j]);               \
        dE[i] += charge * s + acc_kick;                                       \
    }                                                                         \
}                                                                             \
                                                                              \
/* kick.cpp:37-51: out[i] += sum_j V_j sin(omega_j bc_i + phi_j) */           \
void oracle_rf_volt_comp_##SUF(const real *voltage, const real *omega_rf,     \
                               const real *phi_rf, const real *bin_centers,   \
                               int n_rf, int n_bins, real *out)               \
{                                                                             \
    for (int j = 0; j < n_rf; ++j)                                            \
        for (int i = 0; i < n_bins; ++i)                                      \
            out[i] += voltage[j] * SIN(omega_rf[j] * bin_centers[i]           \
                                       + phi_rf[j]);                          \
}                                                                             \
                                                                              \
/* drift.cpp:19-78; solver 0 simple, 1 legacy, 2 exact. */                    \
void oracle_drift_##SUF(real *dt, const real *dE, int solver, real t_rev,     \
                        real length_ratio, real alpha_order, real eta_0,      \
                        real eta_1, real eta_2, real alpha_0, real alpha_1,   \
                        real alpha_2, real beta, real energy, int n)          \
{                                                                             \
    const real T = t_rev * length_ratio;                                      \
    if (solver == 0) {                                                        \
        const real coeff = T * eta_0 / (beta * beta * energy);                \
        for (int i = 0; i < n; ++i) dt[i] += coeff * dE[i];                   \
    } else if (solver == 1) {                                                 \
        /* The reference writes the constants as double literals (1., 2.), \
         * so in its float build these expressions run in double and are   \
         * rounded to float only on assignment; kept verbatim in form.     */ \
        const real c = 1. / (beta * beta * energy);                           \
        const real e0 = eta_0 * c, e1 = eta_1 * c * c, e2 = eta_2 * c * c * c;\
        for (int i = 0; i < n; ++i) {                                         \
            const real d = dE[i];                                             \
            double den;                                                       \
            if (alpha_order == 0) den = 1. - e0 * d;                          \
            else if (alpha_order == 1) den = 1. - e0 * d - e1 * d * d;        \
            else den = 1. - e0 * d - e1 * d * d - e2 * d * d * d;             \
            dt[i] += T * (1. / den - 1.);                                     \
        }                                                                     \
    } else {                                                                  \
        const real ib2 = 1 / (beta * beta);                                   \
        const real ie2 = 1 / (energy * energy);                               \
        for (int i = 0; i < n; ++i) {                                         \
            const real d = dE[i];                                             \
            const real delta = sqrt(1. + ib2 * (d * d * ie2                   \
                                    + 2. * d / energy)) - 1.;                 \
            dt[i] += T * ((1. + alpha_0 * delta                               \
                           + alpha_1 * (delta * delta)                        \
                           + alpha_2 * (delta * delta * delta))               \
                          * (1. + d / energy) / (1. + delta)                  \
                          - 1.);                                              \
        }                                                                     \
    }                                                                         \
}                                                                             \
                                                                              \
/* histogram.cpp:22-73.  The bin is floor((dt-cut_left)*inv_w) rounded to   \
 * float and truncated to int; out-of-range bins (and NaN, which x86        \
 * converts to INT_MIN) are skipped.  The output is overwritten.           */ \
void oracle_histogram_##SUF(const real *dt, real *out, real cut_left,        \
                            real cut_right, int n_slices, int n)             \
{                                                                             \
    const real inv_w = n_slices / (cut_right - cut_left);                     \
    int *h = (int *)calloc((size_t)n_slices, sizeof(int));                    \
    for (int i = 0; i < n; ++i) {                                             \
        const float fb = (float)FLOOR((dt[i] - cut_left) * inv_w);            \
        if (!(fb >= 0.0f) || !(fb < (float)n_slices)) continue;               \
        h[(int)fb] += 1;                                                      \
    }                                                                         \
    for (int k = 0; k < n_slices; ++k) out[k] = (real)h[k];                   \
    free(h);                                                                  \
}                                                                             \
                                                                              \
/* histogram.cpp:75-132: "smooth" deposit, including the reference's weight \
 * convention (bin k gets 0.5-d, its neighbour 0.5+d; these can be < 0).   */ \
void oracle_smooth_histogram_##SUF(const real *dt, real *out, real cut_left, \
                                   real cut_right, int n_slices, int n)      \
{                                                                             \
    const real inv_w = n_slices / (cut_right - cut_left);                     \
    const real w = (cut_right - cut_left) / n_slices;                         \
    const real lo = cut_left + w * (real)0.5;                                 \
    const real hi = cut_right - w * (real)0.5;                                \
    memset(out, 0, sizeof(real) * (size_t)n_slices);                          \
    for (int i = 0; i < n; ++i) {                                             \
        const real a = dt[i];                                                 \
        if (a < lo || a > hi) continue;                                       \
        const real f = (a - cut_left) * inv_w;                                \
        const int k = (int)f;                                                 \
        const real d = f - (real)k;                                           \
        const int k2 = d > (real)0.5 ? (int)(f + (real)1) : (int)(f - (real)1);\
        /* the reference adds the double literal 0.5, so the update runs  \
         * in double even in the float build */                             \
        out[k] = (real)((double)out[k] + 0.5 - (double)d);                    \
        if (k2 >= 0 && k2 < n_slices)                                         \
            out[k2] = (real)((double)out[k2] + 0.5 + (double)d);              \
    }                                                                         \
}                                                                             \
                                                                              \
/* linear_interp_kick.cpp:21-71.  Table slope_k = q (V_{k+1}-V_k) inv_w,    \
 * offset_k = (q V_k - bc_k slope_k) + acc; particles whose bin index      \
 * (as unsigned) is >= n_slices-1 are not kicked.                          */ \
void oracle_linear_interp_kick_##SUF(const real *dt, real *dE,               \
                                     const real *voltage,                     \
                                     const real *bin_centers, real charge,    \
                                     int n_slices, int n, real acc_kick)      \
{                                                                             \
    const real inv_w = (n_slices - 1)                                         \
                       / (bin_centers[n_slices - 1] - bin_centers[0]);        \
    real *slope = (real *)malloc(sizeof(real) * (size_t)(n_slices - 1));      \
    real *offs = (real *)malloc(sizeof(real) * (size_t)(n_slices - 1));       \
    for (int k = 0; k < n_slices - 1; ++k) {                                  \
        slope[k] = charge * (voltage[k + 1] - voltage[k]) * inv_w;            \
        offs[k] = (charge * voltage[k] - bin_centers[k] * slope[k])           \
                  + acc_kick;                                                 \
    }                                                                         \
    for (int i = 0; i < n; ++i) {                                             \
        const real f = FLOOR((dt[i] - bin_centers[0]) * inv_w);               \
        if (!(f >= 0) || !(f < (real)(n_slices - 1))) continue;               \
        const int k = (int)f;                                                 \
        dE[i] += dt[i] * slope[k] + offs[k];                                  \
    }                                                                         \
    free(slope);                                                              \
    free(offs);                                                               \
}                                                                             \
                                                                              \
/* fast_resonator.cpp:19-74: Z += R / (1 + jQ(f/fr - fr/f)), index 0 (DC)   \
 * is left untouched.                                                      */ \
void oracle_fast_resonator_##SUF(real *re, real *im, const real *freq,       \
                                 const real *R, const real *Q,                \
                                 const real *fr, int n_res, int n_f)          \
{                                                                             \
    for (int r = 0; r < n_res; ++r) {                                         \
        const real q2 = Q[r] * Q[r];                                          \
        for (int k = 1; k < n_f; ++k) {                                       \
            const real x = freq[k] / fr[r] - fr[r] / freq[k];                 \
            re[k] += R[r] / (1.0 + q2 * x * x);                               \
            im[k] -= R[r] * (Q[r] * x) / (1.0 + q2 * x * x);                  \
        }                                                                     \
    }                                                                         \
}

/* beam_phase.cpp:6-65 with trapz_const_delta (blondmath.cpp:496-512):     \
 * ratio of the constant-step trapezoids of w p sin(omega bc + phi) and     \
 * w p cos(...), w = exp(alpha bc) (weighted) or 1.                       */
#define DEFINE_BEAM_PHASE(real, SUF, SIN, COS, EXP)                           \
real oracle_beam_phase_##SUF(const real *bc, const real *p, real alpha,      \
                             real omega, real phi, real bin_size, int n,      \
                             int weighted)                                    \
{                                                                             \
    real s = 0, c = 0, s0 = 0, c0 = 0, s1 = 0, c1 = 0;                        \
    for (int i = 0; i < n; ++i) {                                             \
        const real base = weighted ? EXP(alpha * bc[i]) * p[i] : p[i];        \
        const real a = omega * bc[i] + phi;                                   \
        const real fs = base * SIN(a), fc = base * COS(a);                    \
        if (i == 0) { s0 = fs; c0 = fc; }                                     \
        if (i == n - 1) { s1 = fs; c1 = fc; }                                 \
        if (i > 0 && i < n - 1) { s += fs; c += fc; }                         \
    }                                                                         \
    const real ps = (s0 + s1) / 2. + s, pc = (c0 + c1) / 2. + c;              \
    return (bin_size * ps) / (bin_size * pc);                                 \
}

DEFINE_ORACLE(double, f64, sin, floor, sqrt)
DEFINE_ORACLE(float, f32, sinf, floorf, sqrtf)
DEFINE_BEAM_PHASE(double, f64, sin, cos, exp)
DEFINE_BEAM_PHASE(float, f32, sinf, cosf, expf)
