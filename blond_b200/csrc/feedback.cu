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

}  // namespace
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
