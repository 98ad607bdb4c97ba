// Beam phase of the RF beam-phase loop (llrf/beam_feedback.py:276-309):
// cpp_routines/beam_phase.cpp:6-65, the ratio of the sine and cosine
// projections of the (optionally exp(alpha t)-weighted) line density at the
// main RF frequency, each integrated by the trapezoidal rule with constant
// step (blondmath.cpp:496-512):
//     coeff = T[w_i p_i sin(omega_rf bc_i + phi_rf)] / T[w_i p_i cos(...)],
//     T[f] = bin_size ((f_0 + f_{n-1}) / 2 + sum_{i=1}^{n-2} f_i),
//     w_i = exp(alpha bc_i)   (beam_phase)   or 1 (beam_phase_fast).
// One block reduces both sums (the profile is O(10^3-10^5) bins) and writes
// the ratio to device memory, so a caller that stays on the device never
// synchronises.
#include "common.cuh"
#include "feedback.cuh"

#include <algorithm>

namespace bb {
namespace {

constexpr int kPhaseThreads = 1024;

__device__ __forceinline__ double dev_exp(double x) { return exp(x); }
__device__ __forceinline__ float dev_exp(float x) { return expf(x); }
__device__ __forceinline__ void dev_sincos(double x, double* s, double* c) { sincos(x, s, c); }
__device__ __forceinline__ void dev_sincos(float x, float* s, float* c) { sincosf(x, s, c); }

template <typename T, bool WEIGHTED>
__global__ void __launch_bounds__(kPhaseThreads)
beam_phase_kernel(const T* __restrict__ bc, const T* __restrict__ profile, T alpha,
                  T omega_rf, T phi_rf, T bin_size, int n, T* __restrict__ out) {
    T s_sum = 0, c_sum = 0;
    for (int i = threadIdx.x; i < n; i += kPhaseThreads) {
        const T base = WEIGHTED ? dev_exp(alpha * bc[i]) * profile[i] : profile[i];
        T sn, cs;
        dev_sincos(omega_rf * bc[i] + phi_rf, &sn, &cs);
        // interior points weigh 1, the two end points 1/2
        const T w = (i == 0 || i == n - 1) ? T(0.5) : T(1);
        s_sum += w * (base * sn);
        c_sum += w * (base * cs);
    }
    __shared__ T ss[32], sc[32];
    for (int d = 16; d > 0; d >>= 1) {
        s_sum += __shfl_down_sync(0xffffffffu, s_sum, d);
        c_sum += __shfl_down_sync(0xffffffffu, c_sum, d);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        ss[warp] = s_sum;
        sc[warp] = c_sum;
    }
    __syncthreads();
    if (warp == 0) {
        s_sum = ss[lane];  // kPhaseThreads / 32 == 32 warps
        c_sum = sc[lane];
        for (int d = 16; d > 0; d >>= 1) {
            s_sum += __shfl_down_sync(0xffffffffu, s_sum, d);
            c_sum += __shfl_down_sync(0xffffffffu, c_sum, d);
        }
        if (lane == 0) {
            // n == 1: the reference's (f_0 + f_0) / 2 = f_0
            if (n == 1) {
                s_sum *= T(2);
                c_sum *= T(2);
            }
            out[0] = (bin_size * s_sum) / (bin_size * c_sum);
        }
    }
}

template <typename T, bool WEIGHTED>
int beam_phase_impl(const T* bc, const T* profile, T alpha, T omega_rf, T phi_rf, T bin_size,
                    int n_bins, T* coeff, void* stream) {
    clear_error();
    BB_CHECK_ARG(bc && profile && coeff, "beam_phase: null pointer");
    BB_CHECK_SIZE(n_bins >= 1, "beam_phase: n_bins = %d (>= 1 required)", n_bins);
    BB_CHECK_ARG(aligned(bc, sizeof(T)) && aligned(profile, sizeof(T)) &&
                     aligned(coeff, sizeof(T)),
                 "beam_phase: misaligned array");
    beam_phase_kernel<T, WEIGHTED><<<1, kPhaseThreads, 0, as_stream(stream)>>>(
        bc, profile, alpha, omega_rf, phi_rf, bin_size, n_bins, coeff);
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

// ----------------------------------------------------------- engine loop
// Sum of dE[k * sample_dE] over this block's share, one partial per block.
__global__ void __launch_bounds__(256)
fb_dE_kernel(const void* dE, int f32, int64_t n, int sample, double* partials) {
    const int64_t m = (n + sample - 1) / sample;
    double acc = 0.0;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m;
         k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = k * sample;
        acc += f32 ? (double)static_cast<const float*>(dE)[i] : static_cast<const double*>(dE)[i];
    }
    __shared__ double sh[8];
    for (int d = 16; d > 0; d >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, d);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += sh[w];
        partials[blockIdx.x] = t;
    }
}

// Sum of dE[k * sample_dE] after this turn's interpolated kick, computed
// as the particle pass computes it (same table, same expression).  Four
// sampled particles per iteration with their loads issued first: the table
// gather depends on dt, and a chain per particle would leave the pass
// latency-bound.
template <typename E>
__device__ __forceinline__ void lik_apply(double t, E& e, const void* table, double bc0,
                                          double lik_inv_w, double bw, int S) {
    const double f = floor((t - bc0) * lik_inv_w);
    if (!(f >= 0.0 && f < (double)(S - 1))) return;
    const int q = (int)f;
    if constexpr (sizeof(E) == 8) {
        const double2 tb = __ldg(reinterpret_cast<const double2*>(table) + q);
        e += t * tb.x + tb.y;
    } else {
        const float2 tb = __ldg(reinterpret_cast<const float2*>(table) + q);
        const float x = (float)(t - (bc0 + (double)q * bw));
        e += __fmaf_rn(tb.y, x, tb.x);
    }
}

template <typename E>
__global__ void __launch_bounds__(256)
fb_dE_lik_kernel(const double* __restrict__ dt, const E* __restrict__ dE, int64_t n, int sample,
                 const void* table, double bc0, double lik_inv_w, double bw, int S,
                 double* partials) {
    const int64_t m = (n + sample - 1) / sample;
    const int64_t G = (int64_t)gridDim.x * blockDim.x;
    double acc = 0.0;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += 4 * G) {
        double t[4];
        E e[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t idx = k + u * G;
            t[u] = idx < m ? dt[idx * sample] : 0.0;
            e[u] = idx < m ? dE[idx * sample] : E(0);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (k + u * G < m) lik_apply(t[u], e[u], table, bc0, lik_inv_w, bw, S);
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (k + u * G < m) acc += (double)e[u];
    }
    __shared__ double sh[8];
    for (int d = 16; d > 0; d >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, d);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tsum = 0.0;
        for (int w = 0; w < 8; ++w) tsum += sh[w];
        partials[blockIdx.x] = tsum;
    }
}

// One pass per turn: histogram -> profile (histogram cleared) with every
// warp's share of the two projections in phase_partials; the block that
// takes the last ticket (no waiting) sums the shares in index order (and
// SPS_RL's dE partials) and runs the loop; with bump it then advances the
// turn counter (heads without a spectral kernel).  The arguments come by
// value: no pointer chasing on the loop's critical path.
__global__ void __launch_bounds__(kFbThreads)
fb_convert_kernel(const FeedbackArgs a, int* __restrict__ hist, int* __restrict__ ticket,
                  int bump) {
    const long long t = hist ? *a.turn : *a.turn - 1;
    const int S = a.S;
    double* __restrict__ profile = const_cast<double*>(a.profile);
    double s_sum = 0, c_sum = 0;
    const bool active = t >= a.delay;
    FbBins b = {};
    if (active) b = fb_bins(a, t);
    for (int i = blockIdx.x * kFbThreads + threadIdx.x; i < S; i += gridDim.x * kFbThreads) {
        double x;
        if (hist) {
            x = (double)hist[i];
            hist[i] = 0;
            profile[i] = x;
        } else {
            x = profile[i];
        }
        if (active) fb_add(b, i, x, s_sum, c_sum);
    }
    for (int d = 16; d > 0; d >>= 1) {
        s_sum += __shfl_down_sync(0xffffffffu, s_sum, d);
        c_sum += __shfl_down_sync(0xffffffffu, c_sum, d);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int wpb = kFbThreads / 32;
    if (lane == 0) {
        a.phase_partials[2 * (blockIdx.x * wpb + warp)] = s_sum;
        a.phase_partials[2 * (blockIdx.x * wpb + warp) + 1] = c_sum;
        __threadfence();
    }
    __syncthreads();
    int last = 0;
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1) == (int)gridDim.x - 1;
    last = __syncthreads_or(last);
    if (!last || warp != 0) return;
    __threadfence();
    const int parts = gridDim.x * wpb;
    double s = 0, c = 0, dsum = 0;
    for (int q = lane; q < parts; q += 32) {
        s += a.phase_partials[2 * q];
        c += a.phase_partials[2 * q + 1];
    }
    if (a.machine == BLOND_FB_SPS_RL && active)
        for (int q = lane; q < kFbPartials; q += 32) dsum += a.partials[q];
    for (int d = 16; d > 0; d >>= 1) {
        s += __shfl_down_sync(0xffffffffu, s, d);
        c += __shfl_down_sync(0xffffffffu, c, d);
        dsum += __shfl_down_sync(0xffffffffu, dsum, d);
    }
    if (lane == 0) {
        *ticket = 0;  // every block has taken its ticket: ready for the next turn
        fb_turn_end(a, t, s, c, dsum);
        if (bump) *a.turn = t + 1;
    }
}

int convert_grid(int S) {
    const int64_t need = ((int64_t)S + kFbThreads - 1) / kFbThreads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(need, kFbMaxBlocks));
}

}  // namespace

int launch_feedback_dE(const FeedbackArgs& a, cudaStream_t s) {
    if (a.machine == BLOND_FB_SPS_RL) {
        fb_dE_kernel<<<kFbPartials, 256, 0, s>>>(a.dE, a.dE_f32, a.n, a.sample_dE, a.partials);
        BB_LAUNCH_CHECK();
    }
    return BLOND_OK;
}

int launch_feedback_dE_lik(const FeedbackArgs& a, const void* table, double bc0,
                           double lik_inv_w, double bw, cudaStream_t s) {
    if (a.dE_f32)
        fb_dE_lik_kernel<float><<<kFbPartials, 256, 0, s>>>(
            a.dt, static_cast<const float*>(a.dE), a.n, a.sample_dE, table, bc0, lik_inv_w,
            bw, a.S, a.partials);
    else
        fb_dE_lik_kernel<double><<<kFbPartials, 256, 0, s>>>(
            a.dt, static_cast<const double*>(a.dE), a.n, a.sample_dE, table, bc0, lik_inv_w,
            bw, a.S, a.partials);
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

int launch_feedback_turn(const FeedbackArgs& a, int* hist, int* ticket, int bump,
                         cudaStream_t s) {
    fb_convert_kernel<<<convert_grid(a.S), kFbThreads, 0, s>>>(a, hist, ticket, bump);
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

}  // namespace bb

using namespace bb;

extern "C" {

int blond_beam_phase_f64(const double* bin_centers, const double* profile, double alpha,
                         double omega_rf, double phi_rf, double bin_size, int n_bins,
                         double* coeff, void* stream) {
    return beam_phase_impl<double, true>(bin_centers, profile, alpha, omega_rf, phi_rf,
                                         bin_size, n_bins, coeff, stream);
}
int blond_beam_phase_f32(const float* bin_centers, const float* profile, float alpha,
                         float omega_rf, float phi_rf, float bin_size, int n_bins,
                         float* coeff, void* stream) {
    return beam_phase_impl<float, true>(bin_centers, profile, alpha, omega_rf, phi_rf,
                                        bin_size, n_bins, coeff, stream);
}
int blond_beam_phase_fast_f64(const double* bin_centers, const double* profile,
                              double omega_rf, double phi_rf, double bin_size, int n_bins,
                              double* coeff, void* stream) {
    return beam_phase_impl<double, false>(bin_centers, profile, 0.0, omega_rf, phi_rf,
                                          bin_size, n_bins, coeff, stream);
}
int blond_beam_phase_fast_f32(const float* bin_centers, const float* profile, float omega_rf,
                              float phi_rf, float bin_size, int n_bins, float* coeff,
                              void* stream) {
    return beam_phase_impl<float, false>(bin_centers, profile, 0.0f, omega_rf, phi_rf,
                                         bin_size, n_bins, coeff, stream);
}

}  // extern "C"
