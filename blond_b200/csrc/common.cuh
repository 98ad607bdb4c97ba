// Shared helpers for the blond_b200 CUDA library: status codes, the
// thread-local error message, launch geometry and small device utilities.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdarg.h>
#include <math.h>

#include "../../include/blond_b200.h"

namespace bb {

// ---------------------------------------------------------------- errors
void set_error(const char* fmt, ...);
void clear_error();

#define BB_CHECK_ARG(cond, ...)                                              \
    do {                                                                     \
        if (!(cond)) {                                                       \
            ::bb::set_error(__VA_ARGS__);                                    \
            return BLOND_ERR_INVALID_ARGUMENT;                               \
        }                                                                    \
    } while (0)

#define BB_CHECK_SIZE(cond, ...)                                             \
    do {                                                                     \
        if (!(cond)) {                                                       \
            ::bb::set_error(__VA_ARGS__);                                    \
            return BLOND_ERR_SIZE;                                           \
        }                                                                    \
    } while (0)

#define BB_CUDA(call)                                                        \
    do {                                                                     \
        cudaError_t e_ = (call);                                             \
        if (e_ != cudaSuccess) {                                             \
            ::bb::set_error("%s failed: %s (%s:%d)", #call,                  \
                            cudaGetErrorString(e_), __FILE__, __LINE__);     \
            return BLOND_ERR_CUDA;                                           \
        }                                                                    \
    } while (0)

// After a kernel launch: report configuration errors (not asynchronous
// execution errors, which surface at the caller's next synchronisation).
#define BB_LAUNCH_CHECK()                                                    \
    do {                                                                     \
        cudaError_t e_ = cudaGetLastError();                                 \
        if (e_ != cudaSuccess) {                                             \
            ::bb::set_error("kernel launch failed: %s (%s:%d)",              \
                            cudaGetErrorString(e_), __FILE__, __LINE__);     \
            return BLOND_ERR_CUDA;                                           \
        }                                                                    \
    } while (0)

inline bool aligned(const void* p, size_t a) {
    return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0;
}

// ------------------------------------------------------- launch geometry
struct DeviceInfo {
    int device;
    int sm_count;
    int max_smem_optin;  // bytes per block with opt-in
};
// Cached per current device.
const DeviceInfo& device_info();

// Grid for a grid-stride particle loop: a whole number of waves over the
// SMs, never more blocks than there are chunks of work.
inline int particle_grid(int64_t n, int threads, int blocks_per_sm,
                         int items_per_thread = 1) {
    const DeviceInfo& d = device_info();
    int64_t need = (n + (int64_t)threads * items_per_thread - 1) /
                   ((int64_t)threads * items_per_thread);
    int64_t cap = (int64_t)d.sm_count * blocks_per_sm;
    if (need < 1) need = 1;
    return (int)(need < cap ? need : cap);
}

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Programmatic dependent launch (sm_90+): let the grid launched after this
// one on the stream start (it still waits in pdl_wait), and wait for the
// grid before this one to complete and flush its memory.  Both are no-ops
// for a launch without programmatic stream serialization.
__device__ __forceinline__ void pdl_launch_dependents() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// ------------------------------------------------------ device utilities
template <typename T> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };
template <> struct Vec2<int> { using type = int2; };

// sin(x) of an RF phase argument.  The FP64 particle passes spend much of
// their issue slots on this sine, so it is written for the arguments they
// see (|x| up to ~1e3 rad): Cody-Waite reduction by pi (W. J. Cody and
// W. Waite, "Software Manual for the Elementary Functions", 1980) with pi
// split in three parts -- the first two with 30 significant bits, so k P1
// and k P2 are exact for |k| < 2^23 -- to r in [-pi/2, pi/2], then an odd
// polynomial through r^17 (a Chebyshev approximation, coefficients from
// gen_sin_coeffs.py) by Horner's rule in r^2, and sin(x) = (-1)^k sin(r).  No
// branch at all, so a warp's particles stay converged; k is rounded with
// the 1.5 * 2^52 shifter rather than a rounding and a conversion
// instruction.  Within a few units in the last place of the correctly
// rounded sine for |x| < 1e9 (tested against numpy); beyond, the reduction
// is done with fused multiply-adds, each rounding once, so the error grows
// like |x| * 1e-25 (about 1e-13 at 1e12).  Valid for |x| < 2^51 pi (7e15
// rad, hours of beam time at any RF frequency); NaN and inf give NaN.
__device__ __forceinline__ double rf_sin(double x) {
    // k = rint(x / pi): adding and subtracting 1.5 * 2^52 rounds the
    // (rounded) quotient to the nearest integer, ties to even, exactly as
    // rint does for |x / pi| < 2^51, and leaves k's parity in the low bit
    // of the shifted sum
    const double shifter = 6755399441055744.0;  // 1.5 * 2^52
    const double y = __dmul_rn(x, 0.3183098861837907);  // 1 / pi
    const double ks = __dadd_rn(y, shifter);
    const double k = __dsub_rn(ks, shifter);
    double r = fma(-k, 3.1415926553308964, x);       // P1
    r = fma(-k, -1.7411031384001463e-09, r);          // P2
    r = fma(-k, -7.00686879617986e-19, r);            // P3
    const double r2 = r * r;
    // sin r = r + r^3 P(r^2), P the degree-7 Chebyshev approximation on
    // [0, (pi/2)^2] (gen_sin_coeffs.py; error below 1.3e-18)
    double p = 2.7314447669863995e-15;
    p = fma(p, r2, -7.643970296798572e-13);
    p = fma(p, r2, 1.6058977312464087e-10);
    p = fma(p, r2, -2.5052107616996182e-08);
    p = fma(p, r2, 2.7557319219163234e-06);
    p = fma(p, r2, -0.00019841269841254974);
    p = fma(p, r2, 0.008333333333333316);
    p = fma(p, r2, -0.16666666666666666);
    double s = fma(r * r2, p, r);
    return (__double2loint(ks) & 1) ? -s : s;
}

// sin(x) and cos(x) with rf_sin's reduction: cos(x) = (-1)^k cos(r), cos r
// = 1 + r^2 Q(r^2) with Q the degree-8 Chebyshev approximation on
// [0, (pi/2)^2] (gen_sin_coeffs.py; within 1.6e-16 absolute).  Same range
// as rf_sin; no branch.
__device__ __forceinline__ void rf_sincos(double x, double* sp, double* cp) {
    const double shifter = 6755399441055744.0;  // 1.5 * 2^52
    const double y = __dmul_rn(x, 0.3183098861837907);
    const double ks = __dadd_rn(y, shifter);
    const double k = __dsub_rn(ks, shifter);
    double r = fma(-k, 3.1415926553308964, x);
    r = fma(-k, -1.7411031384001463e-09, r);
    r = fma(-k, -7.00686879617986e-19, r);
    const double r2 = r * r;
    double p = 2.7314447669863995e-15;
    p = fma(p, r2, -7.643970296798572e-13);
    p = fma(p, r2, 1.6058977312464087e-10);
    p = fma(p, r2, -2.5052107616996182e-08);
    p = fma(p, r2, 2.7557319219163234e-06);
    p = fma(p, r2, -0.00019841269841254974);
    p = fma(p, r2, 0.008333333333333316);
    p = fma(p, r2, -0.16666666666666666);
    const double s = fma(r * r2, p, r);
    double q = -1.5169166967261124e-16;
    q = fma(q, r2, 4.777404889695354e-14);
    q = fma(q, r2, -1.147069401087498e-11);
    q = fma(q, r2, 2.0876756238770223e-09);
    q = fma(q, r2, -2.7557319217593045e-07);
    q = fma(q, r2, 2.4801587301556646e-05);
    q = fma(q, r2, -0.0013888888888888816);
    q = fma(q, r2, 0.041666666666666664);
    q = fma(q, r2, -0.5);
    const double c = fma(r2, q, 1.0);
    const bool odd = (__double2loint(ks) & 1) != 0;
    *sp = odd ? -s : s;
    *cp = odd ? -c : c;
}

// sin(x) as a float for the F32P64 kick: k = rint(x / pi) by the shifter
// and r = x - k pi with one fused multiply-add in double (exact enough for
// float: |k| (pi - fl(pi)) < 4e-10 below 1e7 rad), then r + r^3 P(r^2) in
// float, P the degree-4 Chebyshev approximation on [0, (pi/2)^2]
// (gen_sin_coeffs.py; within 2 float ulps).  No branch.
__device__ __forceinline__ float rf_sinf(double x) {
    const double shifter = 6755399441055744.0;  // 1.5 * 2^52
    const double ks = __dadd_rn(__dmul_rn(x, 0.3183098861837907), shifter);
    const double k = __dsub_rn(ks, shifter);
    const float r = (float)fma(-k, 3.141592653589793, x);
    const float r2 = r * r;
    float p = -2.408019028621311e-08f;
    p = fmaf(p, r2, 2.75364641311171e-06f);
    p = fmaf(p, r2, -0.00019841086759697646f);
    p = fmaf(p, r2, 0.00833333283662796f);
    p = fmaf(p, r2, -0.1666666716337204f);
    const float s = fmaf(r * r2, p, r);
    return (__double2loint(ks) & 1) ? -s : s;
}

__device__ __forceinline__ double dev_sin(double x) { return rf_sin(x); }
__device__ __forceinline__ float dev_sin(float x) { return sinf(x); }
__device__ __forceinline__ double dev_floor(double x) { return floor(x); }
__device__ __forceinline__ float dev_floor(float x) { return floorf(x); }
__device__ __forceinline__ double dev_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float dev_sqrt(float x) { return sqrtf(x); }

// Plain IEEE multiply / subtract that the compiler may not fuse into an FMA.
// The histogram bin expression floor((dt - cut_left) * inv_w) must round
// exactly like the reference's C++ for bit-exact counts.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }

// Bin centre i of S slices over [lo, hi] as the reference's Profile forms
// it (beam/profile.py:207-211): edges = numpy.linspace(lo, hi, S + 1),
// which numpy evaluates as i * step + lo with step = (hi - lo) / S and the
// last edge set to hi; centre i = (edge_i + edge_{i+1}) / 2.  Every
// operation rounds on its own (no contraction), on the host and the device,
// so both give numpy's bits.
__host__ __device__ inline double linspace_edge(double lo, double hi, int S, int i) {
    if (i >= S) return hi;
#ifdef __CUDA_ARCH__
    const double step = __ddiv_rn(__dsub_rn(hi, lo), (double)S);
    return __dadd_rn(__dmul_rn((double)i, step), lo);
#else
    const volatile double step = (hi - lo) / (double)S;
    const volatile double x = (double)i * step;
    return x + lo;
#endif
}
__host__ __device__ inline double linspace_centre(double lo, double hi, int S, int i) {
#ifdef __CUDA_ARCH__
    return __dmul_rn(__dadd_rn(linspace_edge(lo, hi, S, i), linspace_edge(lo, hi, S, i + 1)),
                     0.5);
#else
    const volatile double sum = linspace_edge(lo, hi, S, i) + linspace_edge(lo, hi, S, i + 1);
    return sum / 2;
#endif
}

// Entry k of the induced kick's interpolation table from the voltages at bin
// centres k and k+1 (linear_interp_kick.cpp:44-47):
//   slope  = charge (V_{k+1} - V_k) inv_w
//   offset = (charge V_k - bc_k slope) + acc
// every operation rounded on its own, so the head kernel that writes the
// table and a particle pass that forms entries from a voltage-only copy give
// the same bits.
__device__ __forceinline__ double2 lik_entry(double v0, double v1, double bc, double charge,
                                             double inv_w, double acc) {
    const double slope = __dmul_rn(__dmul_rn(charge, __dsub_rn(v1, v0)), inv_w);
    const double offset = __dadd_rn(__dsub_rn(__dmul_rn(charge, v0), __dmul_rn(bc, slope)), acc);
    return make_double2(slope, offset);
}

// The same with no acceleration kick in the offset (the fused turn applies
// it with the RF kick): the "+ 0" is left out, which changes nothing but
// the sign of a zero offset.  The head's table and the shared-table pass
// both use this form, so they agree bit for bit.
__device__ __forceinline__ double2 lik_entry0(double v0, double v1, double bc, double charge,
                                              double inv_w) {
    const double slope = __dmul_rn(__dmul_rn(charge, __dsub_rn(v1, v0)), inv_w);
    const double offset = __dsub_rn(__dmul_rn(charge, v0), __dmul_rn(bc, slope));
    return make_double2(slope, offset);
}

// ------------------------------------------------------ smooth deposit weights
// histogram.cpp:75-132.  Weights of a particle at f = (dt-cut_left)*inv_w,
// k = (int)f, d = f-k: bin k gets 0.5-d; bin k+1 (d > 0.5) or k-1 (else)
// gets 0.5+d.  The bmath kernel accumulates them with floating-point
// atomics (the summation order, not the set of terms, differs from the
// reference's); the fused turn in 64-bit fixed point (engine.cu).
template <typename T>
__device__ __forceinline__ void smooth_weights(T a, T cut_left, T inv_w, T lo,
                                               T hi, int S, int& k, int& k2,
                                               double& w1, double& w2) {
    k = -1;
    k2 = -1;
    if (!(a >= lo && a <= hi)) return;  // also rejects NaN
    const T f = (a - cut_left) * inv_w;
    k = (int)f;
    const T d = f - (T)k;
    k2 = d > T(0.5) ? (int)((double)f + 1.0) : (int)((double)f - 1.0);
    w1 = 0.5 - (double)d;
    w2 = 0.5 + (double)d;
    if (k < 0 || k >= S) k = -1;
    if (k2 < 0 || k2 >= S) k2 = -1;
}

// ------------------------------------------------------------ drift solvers
// drift.cpp:29-76.  The expressions of the 'legacy' and 'exact' solvers
// cancel (1/(1-x)-1 with x ~ 1e-6), so they are evaluated operation by
// operation without FMA contraction, in the reference's order and with its
// C promotion rules: the constants are double literals (1., 2.), so in the
// float build the marked sub-expressions run in double and are rounded to
// the element type only where the reference assigns them.  This makes the
// result bit-identical to the reference compiled without -ffast-math.
template <typename T>
__device__ __forceinline__ T drift_simple(T dt, T d, T coeff) {
    return add_rn(dt, mul_rn(coeff, d));
}

template <typename T>
__device__ __forceinline__ T drift_legacy(T dt, T d, T Tr, T e0, T e1, T e2, int order) {
    double den = __dsub_rn(1.0, (double)mul_rn(e0, d));
    if (order >= 1) den = __dsub_rn(den, (double)mul_rn(mul_rn(e1, d), d));
    if (order >= 2) den = __dsub_rn(den, (double)mul_rn(mul_rn(mul_rn(e2, d), d), d));
    const double inc = __dmul_rn((double)Tr, __dsub_rn(__ddiv_rn(1.0, den), 1.0));
    return (T)__dadd_rn((double)dt, inc);
}

template <typename T>
__device__ __forceinline__ T drift_exact(T dt, T d, T Tr, T ib2, T ie2, T a0, T a1,
                                         T a2, T energy) {
    const double inner = __dadd_rn((double)mul_rn(mul_rn(d, d), ie2),
                                   __ddiv_rn(__dmul_rn(2.0, (double)d), (double)energy));
    const T delta = (T)__dsub_rn(__dsqrt_rn(__dadd_rn(1.0, __dmul_rn((double)ib2, inner))),
                                 1.0);
    double num = __dadd_rn(1.0, (double)mul_rn(a0, delta));
    num = __dadd_rn(num, (double)mul_rn(a1, mul_rn(delta, delta)));
    num = __dadd_rn(num, (double)mul_rn(a2, mul_rn(mul_rn(delta, delta), delta)));
    const double f = __dsub_rn(
        __ddiv_rn(__dmul_rn(num, __dadd_rn(1.0, (double)div_rn(d, energy))),
                  __dadd_rn(1.0, (double)delta)),
        1.0);
    return (T)__dadd_rn((double)dt, __dmul_rn((double)Tr, f));
}

}  // namespace bb
