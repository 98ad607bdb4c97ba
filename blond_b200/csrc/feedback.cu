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

// first index with bc >= x (count of bc < x), bc increasing
__device__ int fb_lower(const double* bc, int S, double x) {
    int lo = 0, hi = S;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (bc[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo;
}
// first index with bc > x
__device__ int fb_upper(const double* bc, int S, double x) {
    int lo = 0, hi = S;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (bc[mid] <= x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(kPhaseThreads) feedback_kernel(FeedbackArgs a) {
    __shared__ int range[2];
    __shared__ double ss[32], sc[32], sd[32];
    const long long t = *a.turn - 1;
    const int nr = a.n_rf;
    const int cols = FB_COLS + 2 * nr;
    const double* row = a.table + (size_t)t * cols;
    const double* next = a.table + (size_t)(t + 1) * cols;
    const bool active = t >= a.delay;
    const double omega = a.om[(size_t)t * nr], phi = a.ph[(size_t)t * nr];
    if (threadIdx.x == 0) {
        int start = 0, stop = a.S;
        if (a.machine == BLOND_FB_SPS_F) {
            // beam_feedback.py:326-334: window from time_offset and alpha
            if (a.alpha != 0.0) {
                const double lo = a.time_offset - M_PI / omega;
                const double hi = -1 / a.alpha + a.time_offset - 2 * M_PI / omega;
                start = fb_lower(a.bc, a.S, lo);
                stop = max(start, fb_upper(a.bc, a.S, hi));
            }
        } else if (a.has_time_offset) {
            start = fb_lower(a.bc, a.S, a.time_offset);
        }
        range[0] = start;
        range[1] = stop;
    }
    __syncthreads();
    const int start = range[0], stop = range[1], n = stop - start;
    const bool weighted = a.machine != BLOND_FB_SPS_F;
    double s_sum = 0, c_sum = 0, d_sum = 0;
    if (active) {
        for (int k = threadIdx.x; k < n; k += kPhaseThreads) {
            const int i = start + k;
            const double base = weighted ? exp(a.alpha * a.bc[i]) * a.profile[i] : a.profile[i];
            double sn, cs;
            sincos(omega * a.bc[i] + phi, &sn, &cs);
            const double w = (k == 0 || k == n - 1) ? 0.5 : 1.0;
            s_sum += w * (base * sn);
            c_sum += w * (base * cs);
        }
        if (a.machine == BLOND_FB_SPS_RL)
            for (int k = threadIdx.x; k < kFbPartials; k += kPhaseThreads) d_sum += a.partials[k];
    }
    for (int d = 16; d > 0; d >>= 1) {
        s_sum += __shfl_down_sync(0xffffffffu, s_sum, d);
        c_sum += __shfl_down_sync(0xffffffffu, c_sum, d);
        d_sum += __shfl_down_sync(0xffffffffu, d_sum, d);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        ss[warp] = s_sum;
        sc[warp] = c_sum;
        sd[warp] = d_sum;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    s_sum = c_sum = d_sum = 0;
    for (int w = 0; w < kPhaseThreads / 32; ++w) {
        s_sum += ss[w];
        c_sum += sc[w];
        d_sum += sd[w];
    }
    double* st = a.state;
    double domega = st[FBS_DOMEGA_RF];
    if (active) {
        if (n == 1) {
            s_sum *= 2;
            c_sum *= 2;
        }
        const double coeff = n > 0 ? (a.bin_size * s_sum) / (a.bin_size * c_sum) : nan("");
        const double phi_beam = atan(coeff) + M_PI;
        const double dphi = phi_beam - row[FBT_PHI_S];
        const double om_off = omega - row[FB_COLS];  // omega_rf - omega_rf_d, main system
        switch (a.machine) {
        case BLOND_FB_LHC: {  // beam_feedback.py:516-565
            const double dphi_rf = st[FBS_DPHI_RF];
            const double la = row[FBT_LHC_A], lt = row[FBT_LHC_T];
            domega = -a.gain * dphi - a.gain2 * (st[FBS_LHC_Y] + la * (dphi_rf + 0.0));
            st[FBS_LHC_Y] = (1 - lt) * st[FBS_LHC_Y] + (1 - la) * lt * (dphi_rf + 0.0);
            break;
        }
        case BLOND_FB_LHC_F:  // beam_feedback.py:432-458
            domega = -a.gain * dphi - a.gain2 * (om_off + 0.0);
            break;
        case BLOND_FB_SPS_F:  // beam_feedback.py:460-479
            domega = -a.gain * dphi + -a.gain2 * om_off;
            break;
        case BLOND_FB_SPS_RL: {  // beam_feedback.py:370-391, 481-514
            const int64_t m = (a.n + a.sample_dE - 1) / a.sample_dE;
            const double avg = d_sum / (double)m;
            const double drho = row[FBT_ALPHA0] * a.ring_radius * avg /
                                (row[FBT_BETA] * row[FBT_BETA] * row[FBT_ENERGY]);
            const double sgn = row[FBT_ETA0] > 0 ? 1.0 : (row[FBT_ETA0] < 0 ? -1.0 : 0.0);
            st[FBS_AVG_DE] = avg;
            st[FBS_DRHO] = drho;
            domega = -a.gain * dphi + -sgn * a.gain2 * (0.0 - drho) / a.ring_radius;
            break;
        }
        case BLOND_FB_PSB: {  // beam_feedback.py:567-622
            st[FBS_DPHI_SUM] += dphi;
            const int pc = (int)st[FBS_PL_COUNTER];
            if (pc < a.n_on_time && (double)t == a.on_time[pc] && t >= a.delay) {
                const double prev = a.on_time[pc > 0 ? pc - 1 : a.n_on_time - 1];
                const double av = st[FBS_DPHI_SUM] / (a.on_time[pc] - prev);
                st[FBS_DPHI_AV] = av;
                st[FBS_DOMEGA_PL] = 0.99803799 * st[FBS_DOMEGA_PL] +
                                    row[FBT_GAIN] * (0.99901903 * av - 0.99901003 * st[FBS_DPHI_AV_PREV]);
                st[FBS_DPHI_AV_PREV] = av;
                st[FBS_DPHI_SUM] = 0.0;
                const double g = row[FBT_GAMMA];
                const double dr = om_off / (row[FB_COLS] * (1.0 / (row[FBT_ALPHA0] * (g * g)) - 1.0));
                st[FBS_DR] = dr;
                st[FBS_DOMEGA_RL] = st[FBS_DOMEGA_RL] + row[FBT_GAIN2A] * (dr - st[FBS_DR_PREV]) +
                                    row[FBT_GAIN2B] * dr;
                st[FBS_DR_PREV] = dr;
                st[FBS_PL_COUNTER] = pc + 1;
            }
            domega = -st[FBS_DOMEGA_PL] - st[FBS_DOMEGA_RL];
            break;
        }
        }
        st[FBS_PHI_BEAM] = phi_beam;
        st[FBS_DPHI] = dphi;
        st[FBS_DOMEGA_RF] = domega;
        // BeamFeedback.track: next turn's frequency of every system
        const double* h1 = next + FB_COLS + nr;
        for (int j = 0; j < nr; ++j) a.om[(size_t)(t + 1) * nr + j] += domega * h1[j] / h1[0];
    }
    // RingAndRFTracker.track (tracker.py:553-565): accumulated phase offset
    bool any = false;
    for (int j = 0; j < nr; ++j) {
        const double od = next[FB_COLS + j], h = next[FB_COLS + nr + j];
        st[FBS_DPHI_RF + j] += 2.0 * M_PI * h * (a.om[(size_t)(t + 1) * nr + j] - od) / od;
        any = any || st[FBS_DPHI_RF + j] != 0.0;
    }
    if (any)
        for (int j = 0; j < nr; ++j) a.ph[(size_t)(t + 1) * nr + j] += st[FBS_DPHI_RF + j];
    if (a.trace) {
        a.trace[t * 3 + 0] = st[FBS_PHI_BEAM];
        a.trace[t * 3 + 1] = st[FBS_DPHI];
        a.trace[t * 3 + 2] = st[FBS_DOMEGA_RF];
    }
}

}  // namespace

int launch_feedback(const FeedbackArgs& a, cudaStream_t s) {
    if (a.machine == BLOND_FB_SPS_RL) {
        fb_dE_kernel<<<kFbPartials, 256, 0, s>>>(a.dE, a.dE_f32, a.n, a.sample_dE, a.partials);
        BB_LAUNCH_CHECK();
    }
    feedback_kernel<<<1, kPhaseThreads, 0, s>>>(a);
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
