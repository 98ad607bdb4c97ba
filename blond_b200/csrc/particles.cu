// bmath-level particle kernels: RF kick, drift, slicing (plain and smooth),
// linear interpolated kick, RF voltage table, resonator impedance.
//
// One launch per call, asynchronous on the caller's stream, in-place on the
// caller's device arrays -- the contract of the reference's ctypes-bound
// libblond routines (blond/utils/butils_wrap_cpp.py:835-989), but each
// routine here is a single HBM pass sized to the B200 (grid = waves of the
// 148 SMs, coalesced loads, shared-memory-privatised histograms).
#include "common.cuh"

#include <mutex>
#include <string.h>

namespace bb {

// ------------------------------------------------------------------ errors
static thread_local char g_err[512] = {0};

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}
void clear_error() { g_err[0] = 0; }

// ------------------------------------------------------------ device info
const DeviceInfo& device_info() {
    static DeviceInfo cache[64];
    static bool valid[64] = {false};
    static std::mutex mu;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    std::lock_guard<std::mutex> lock(mu);
    if (!valid[dev]) {
        DeviceInfo d;
        d.device = dev;
        if (cudaDeviceGetAttribute(&d.sm_count, cudaDevAttrMultiProcessorCount,
                                   dev) != cudaSuccess)
            d.sm_count = 148;
        if (cudaDeviceGetAttribute(&d.max_smem_optin,
                                   cudaDevAttrMaxSharedMemoryPerBlockOptin,
                                   dev) != cudaSuccess)
            d.max_smem_optin = 48 * 1024;
        cache[dev] = d;
        valid[dev] = true;
    }
    return cache[dev];
}

// Shared memory the histogram kernels may claim: the opt-in maximum less a
// little for static use.
static int histogram_smem_budget() {
    return device_info().max_smem_optin - 1024;
}

constexpr int kThreads = 512;
constexpr int kMaxRf = 64;

// ------------------------------------------------------------ RF kick
template <typename T>
__global__ void __launch_bounds__(kThreads)
kick_kernel(const T* __restrict__ dt, T* __restrict__ dE, int n_rf, T charge,
            const T* __restrict__ voltage, const T* __restrict__ omega,
            const T* __restrict__ phi, int64_t n, T acc) {
    __shared__ T sv[kMaxRf], so[kMaxRf], sp[kMaxRf];
    for (int j = threadIdx.x; j < n_rf; j += blockDim.x) {
        sv[j] = voltage[j];
        so[j] = omega[j];
        sp[j] = phi[j];
    }
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += stride) {
        const T t = dt[i];
        T s = 0;
        for (int j = 0; j < n_rf; ++j) s += sv[j] * dev_sin(so[j] * t + sp[j]);
        dE[i] += charge * s + acc;
    }
}

template <typename T>
static int kick_impl(const T* dt, T* dE, int n_rf, T charge, const T* V,
                     const T* om, const T* ph, int64_t n, T acc,
                     void* stream) {
    BB_CHECK_ARG(n >= 0, "kick: negative particle count");
    BB_CHECK_SIZE(n_rf >= 0 && n_rf <= kMaxRf, "kick: n_rf=%d outside [0, %d]",
                  n_rf, kMaxRf);
    if (n == 0) return BLOND_OK;
    BB_CHECK_ARG(dt && dE, "kick: null particle array");
    BB_CHECK_ARG(n_rf == 0 || (V && om && ph), "kick: null RF array");
    const int grid = particle_grid(n, kThreads, 4);
    kick_kernel<T><<<grid, kThreads, 0, as_stream(stream)>>>(
        dt, dE, n_rf, charge, V, om, ph, n, acc);
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

// ------------------------------------------------------- RF voltage table
template <typename T>
__global__ void rf_volt_comp_kernel(const T* __restrict__ voltage,
                                    const T* __restrict__ omega,
                                    const T* __restrict__ phi,
                                    const T* __restrict__ bc, int n_rf,
                                    int64_t n_bins, T* __restrict__ out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
         i < n_bins; i += stride) {
        T acc = out[i];
        const T b = bc[i];
        for (int j = 0; j < n_rf; ++j) acc += voltage[j] * dev_sin(omega[j] * b + phi[j]);
        out[i] = acc;
    }
}

template <typename T>
static int rf_volt_comp_impl(const T* V, const T* om, const T* ph,
                             const T* bc, int n_rf, int64_t n_bins, T* out,
                             void* stream) {
    BB_CHECK_ARG(n_bins >= 0 && n_rf >= 0, "rf_volt_comp: negative size");
    if (n_bins == 0 || n_rf == 0) return BLOND_OK;
    BB_CHECK_ARG(V && om && ph && bc && out, "rf_volt_comp: null pointer");
    const int grid = particle_grid(n_bins, 256, 4);
    rf_volt_comp_kernel<T><<<grid, 256, 0, as_stream(stream)>>>(V, om, ph, bc,
                                                                n_rf, n_bins, out);
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

// ------------------------------------------------------------ drift
struct DriftCoeffs {
    double T;       // t_rev * length_ratio
    double simple;  // T * eta_0 / (beta^2 E)
    double e0, e1, e2;  // legacy: eta_i / (beta^2 E)^(i+1)
    double ib2, ie2, inv_e;  // exact: 1/beta^2, 1/E^2
    double a0, a1, a2, energy;
    int order;
};

template <typename T, int SOLVER>
__global__ void __launch_bounds__(kThreads)
drift_kernel(T* __restrict__ dt, const T* __restrict__ dE, int64_t n,
             T Tr, T c_simple, T e0, T e1, T e2, T ib2, T ie2, T a0, T a1,
             T a2, T energy, int order) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += stride) {
        const T d = dE[i];
        if (SOLVER == BLOND_SOLVER_SIMPLE)
            dt[i] = drift_simple<T>(dt[i], d, c_simple);
        else if (SOLVER == BLOND_SOLVER_LEGACY)
            dt[i] = drift_legacy<T>(dt[i], d, Tr, e0, e1, e2, order);
        else
            dt[i] = drift_exact<T>(dt[i], d, Tr, ib2, ie2, a0, a1, a2, energy);
    }
}

template <typename T>
static int drift_impl(T* dt, const T* dE, int solver, T t_rev, T length_ratio,
                      T alpha_order, T eta_0, T eta_1, T eta_2, T alpha_0,
                      T alpha_1, T alpha_2, T beta, T energy, int64_t n,
                      void* stream) {
    BB_CHECK_ARG(n >= 0, "drift: negative particle count");
    BB_CHECK_ARG(solver >= 0 && solver <= 2, "drift: solver %d not in {0,1,2}",
                 solver);
    if (n == 0) return BLOND_OK;
    BB_CHECK_ARG(dt && dE, "drift: null particle array");
    // Coefficients in the element type, with the reference's expression
    // order (drift.cpp:33-56).
    const T Tr = t_rev * length_ratio;
    const T c_simple = Tr * eta_0 / (beta * beta * energy);
    // `1. / (...)` in the reference: a double division rounded to T
    const T coeff = (T)(1.0 / (double)(beta * beta * energy));
    const T e0 = eta_0 * coeff, e1 = eta_1 * coeff * coeff,
            e2 = eta_2 * coeff * coeff * coeff;
    const T ib2 = T(1) / (beta * beta), ie2 = T(1) / (energy * energy);
    const int order = alpha_order == T(0) ? 0 : (alpha_order == T(1) ? 1 : 2);
    const int grid = particle_grid(n, kThreads, 4);
    cudaStream_t s = as_stream(stream);
    if (solver == 0)
        drift_kernel<T, 0><<<grid, kThreads, 0, s>>>(dt, dE, n, Tr, c_simple, e0, e1, e2,
                                                     ib2, ie2, alpha_0, alpha_1, alpha_2,
                                                     energy, order);
    else if (solver == 1)
        drift_kernel<T, 1><<<grid, kThreads, 0, s>>>(dt, dE, n, Tr, c_simple, e0, e1, e2,
                                                     ib2, ie2, alpha_0, alpha_1, alpha_2,
                                                     energy, order);
    else
        drift_kernel<T, 2><<<grid, kThreads, 0, s>>>(dt, dE, n, Tr, c_simple, e0, e1, e2,
                                                     ib2, ie2, alpha_0, alpha_1, alpha_2,
                                                     energy, order);
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

// ------------------------------------------------------------ histogram
// Bin of a particle exactly as histogram.cpp:42-55: floor((dt - cut_left)
// * inv_w) with no FMA contraction, kept iff 0 <= bin < n_slices.  NaN and
// out-of-range coordinates give -1 (skipped).
template <typename T>
__device__ __forceinline__ int slice_bin(T x, T cut_left, T inv_w, int S) {
    const T f = dev_floor(mul_rn(sub_rn(x, cut_left), inv_w));
    return (f >= T(0) && f < T(S)) ? (int)f : -1;
}

// Shared-memory-privatised integer histogram.  With WARP_AGG the lanes of a
// warp that hit the same bin are merged by __match_any_sync so one lane adds
// the popcount -- worthwhile when few bins take most particles.
template <typename T, bool WARP_AGG>
__global__ void __launch_bounds__(kThreads)
histogram_smem_kernel(const T* __restrict__ dt, T* __restrict__ out,
                      T cut_left, T inv_w, int S, int64_t n) {
    extern __shared__ int sh[];
    for (int k = threadIdx.x; k < S; k += blockDim.x) sh[k] = 0;
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31;
    // whole warps iterate together so __match_any_sync sees all 32 lanes
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31);
         base < n; base += stride) {
        const int64_t i = base + lane;
        const int b = i < n ? slice_bin<T>(dt[i], cut_left, inv_w, S) : -1;
        if (WARP_AGG) {
            const unsigned peers = __match_any_sync(0xffffffffu, b);
            if (b >= 0 && lane == __ffs(peers) - 1) atomicAdd(&sh[b], __popc(peers));
        } else if (b >= 0) {
            atomicAdd(&sh[b], 1);
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < S; k += blockDim.x) {
        const int c = sh[k];
        if (c) atomicAdd(&out[k], (T)c);
    }
}

// Fallback for profiles too large to privatise: global atomics on the
// (exactly representable) integer counts.
template <typename T>
__global__ void histogram_global_kernel(const T* __restrict__ dt,
                                        T* __restrict__ out, T cut_left,
                                        T inv_w, int S, int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += stride) {
        const int b = slice_bin<T>(dt[i], cut_left, inv_w, S);
        if (b >= 0) atomicAdd(&out[b], T(1));
    }
}

template <typename T>
static int histogram_impl(const T* dt, T* out, T cut_left, T cut_right,
                          int S, int64_t n, void* stream) {
    BB_CHECK_ARG(n >= 0, "histogram: negative particle count");
    BB_CHECK_SIZE(S >= 1, "histogram: n_slices=%d must be >= 1", S);
    BB_CHECK_ARG(out, "histogram: null profile");
    BB_CHECK_ARG(n == 0 || dt, "histogram: null dt");
    cudaStream_t s = as_stream(stream);
    BB_CUDA(cudaMemsetAsync(out, 0, sizeof(T) * (size_t)S, s));
    if (n == 0) return BLOND_OK;
    // histogram.cpp:30: int / real_t in the element type
    const T inv_w = (T)S / (cut_right - cut_left);
    const size_t smem = sizeof(int) * (size_t)S;
    if ((int64_t)smem <= histogram_smem_budget()) {
        // one or two resident blocks per SM depending on the table size
        const int per_sm = smem <= 96 * 1024 ? 2 : 1;
        const int grid = particle_grid(n, kThreads, per_sm);
        if (S <= 2048) {
            BB_CUDA(cudaFuncSetAttribute(histogram_smem_kernel<T, true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem));
            histogram_smem_kernel<T, true><<<grid, kThreads, smem, s>>>(dt, out, cut_left,
                                                                        inv_w, S, n);
        } else {
            BB_CUDA(cudaFuncSetAttribute(histogram_smem_kernel<T, false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem));
            histogram_smem_kernel<T, false><<<grid, kThreads, smem, s>>>(dt, out, cut_left,
                                                                         inv_w, S, n);
        }
    } else {
        const int grid = particle_grid(n, 256, 8);
        histogram_global_kernel<T><<<grid, 256, 0, s>>>(dt, out, cut_left, inv_w, S, n);
    }
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

// ------------------------------------------------------- smooth histogram
// (smooth_weights: common.cuh)
template <typename T>
__global__ void __launch_bounds__(kThreads)
smooth_histogram_kernel(const T* __restrict__ dt, T* __restrict__ out,
                        T cut_left, T inv_w, T lo, T hi, int S, int64_t n,
                        bool use_smem) {
    extern __shared__ unsigned char raw[];
    T* sh = reinterpret_cast<T*>(raw);
    if (use_smem) {
        for (int k = threadIdx.x; k < S; k += blockDim.x) sh[k] = 0;
        __syncthreads();
    }
    T* dst = use_smem ? sh : out;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += stride) {
        int k, k2;
        double w1 = 0, w2 = 0;
        smooth_weights<T>(dt[i], cut_left, inv_w, lo, hi, S, k, k2, w1, w2);
        if (k >= 0) atomicAdd(&dst[k], (T)w1);
        if (k2 >= 0) atomicAdd(&dst[k2], (T)w2);
    }
    if (use_smem) {
        __syncthreads();
        for (int k = threadIdx.x; k < S; k += blockDim.x) {
            const T c = sh[k];
            if (c != T(0)) atomicAdd(&out[k], c);
        }
    }
}

template <typename T>
static int smooth_histogram_impl(const T* dt, T* out, T cut_left, T cut_right,
                                 int S, int64_t n, void* stream) {
    BB_CHECK_ARG(n >= 0, "smooth_histogram: negative particle count");
    BB_CHECK_SIZE(S >= 1, "smooth_histogram: n_slices=%d must be >= 1", S);
    BB_CHECK_ARG(out, "smooth_histogram: null profile");
    BB_CHECK_ARG(n == 0 || dt, "smooth_histogram: null dt");
    cudaStream_t s = as_stream(stream);
    BB_CUDA(cudaMemsetAsync(out, 0, sizeof(T) * (size_t)S, s));
    if (n == 0) return BLOND_OK;
    const T inv_w = (T)S / (cut_right - cut_left);
    const T w = (cut_right - cut_left) / (T)S;
    const T lo = cut_left + w * T(0.5);
    const T hi = cut_right - w * T(0.5);
    const size_t smem = sizeof(T) * (size_t)S;
    const bool use_smem = (int64_t)smem <= histogram_smem_budget();
    const int grid = particle_grid(n, kThreads, use_smem && smem > 96 * 1024 ? 1 : 2);
    BB_CUDA(cudaFuncSetAttribute(smooth_histogram_kernel<T>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 use_smem ? (int)smem : 0));
    smooth_histogram_kernel<T><<<grid, kThreads, use_smem ? smem : 0, s>>>(
        dt, out, cut_left, inv_w, lo, hi, S, n, use_smem);
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

// ------------------------------------------------- linear interpolated kick
// linear_interp_kick.cpp:21-71.  The per-slice slope/offset of the
// reference's table are recomputed at the gathered slice with the same
// expressions, so no table buffer is needed.
template <typename T>
__global__ void __launch_bounds__(kThreads)
lik_kernel(const T* __restrict__ dt, T* __restrict__ dE,
           const T* __restrict__ V, const T* __restrict__ bc, T charge, int S,
           int64_t n, T acc) {
    const T bc0 = bc[0];
    const T inv_w = (T)(S - 1) / (bc[S - 1] - bc0);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += stride) {
        const T t = dt[i];
        const T f = dev_floor((t - bc0) * inv_w);
        if (!(f >= T(0) && f < T(S - 1))) continue;
        const int k = (int)f;
        const T v0 = __ldg(V + k), v1 = __ldg(V + k + 1);
        const T slope = charge * (v1 - v0) * inv_w;
        const T offset = (charge * v0 - __ldg(bc + k) * slope) + acc;
        dE[i] += t * slope + offset;
    }
}

template <typename T>
static int lik_impl(const T* dt, T* dE, const T* V, const T* bc, T charge,
                    int S, int64_t n, T acc, void* stream) {
    BB_CHECK_ARG(n >= 0, "linear_interp_kick: negative particle count");
    BB_CHECK_SIZE(S >= 2, "linear_interp_kick: n_slices=%d must be >= 2", S);
    if (n == 0) return BLOND_OK;
    BB_CHECK_ARG(dt && dE && V && bc, "linear_interp_kick: null pointer");
    const int grid = particle_grid(n, kThreads, 4);
    lik_kernel<T><<<grid, kThreads, 0, as_stream(stream)>>>(dt, dE, V, bc, charge, S,
                                                            n, acc);
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

// ------------------------------------------------------- resonator impedance
__global__ void fast_resonator_kernel(double* __restrict__ re,
                                      double* __restrict__ im,
                                      const double* __restrict__ f,
                                      const double* __restrict__ R,
                                      const double* __restrict__ Q,
                                      const double* __restrict__ fr, int nr,
                                      int64_t nf) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = 1 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nf;
         k += stride) {
        double a = re[k], b = im[k];
        const double fk = f[k];
        for (int r = 0; r < nr; ++r) {
            const double q2 = Q[r] * Q[r];
            const double x = fk / fr[r] - fr[r] / fk;
            a += R[r] / (1.0 + q2 * x * x);
            b -= R[r] * (Q[r] * x) / (1.0 + q2 * x * x);
        }
        re[k] = a;
        im[k] = b;
    }
}

}  // namespace bb

using namespace bb;

// ====================================================================== C ABI
extern "C" {

const char* blond_b200_last_error(void) { return g_err; }
int blond_b200_version(void) { return 100; }
int blond_b200_max_smem_slices(void) { return histogram_smem_budget() / 4; }

int blond_kick_f64(const double* dt, double* dE, int n_rf, double charge,
                   const double* V, const double* om, const double* ph,
                   int64_t n, double acc, void* stream) {
    return kick_impl<double>(dt, dE, n_rf, charge, V, om, ph, n, acc, stream);
}
int blond_kick_f32(const float* dt, float* dE, int n_rf, float charge,
                   const float* V, const float* om, const float* ph, int64_t n,
                   float acc, void* stream) {
    return kick_impl<float>(dt, dE, n_rf, charge, V, om, ph, n, acc, stream);
}

int blond_rf_volt_comp_f64(const double* V, const double* om, const double* ph,
                           const double* bc, int n_rf, int64_t n_bins,
                           double* out, void* stream) {
    return rf_volt_comp_impl<double>(V, om, ph, bc, n_rf, n_bins, out, stream);
}
int blond_rf_volt_comp_f32(const float* V, const float* om, const float* ph,
                           const float* bc, int n_rf, int64_t n_bins,
                           float* out, void* stream) {
    return rf_volt_comp_impl<float>(V, om, ph, bc, n_rf, n_bins, out, stream);
}

int blond_drift_f64(double* dt, const double* dE, int solver, double t_rev,
                    double length_ratio, double alpha_order, double eta_0,
                    double eta_1, double eta_2, double alpha_0, double alpha_1,
                    double alpha_2, double beta, double energy, int64_t n,
                    void* stream) {
    return drift_impl<double>(dt, dE, solver, t_rev, length_ratio, alpha_order,
                              eta_0, eta_1, eta_2, alpha_0, alpha_1, alpha_2,
                              beta, energy, n, stream);
}
int blond_drift_f32(float* dt, const float* dE, int solver, float t_rev,
                    float length_ratio, float alpha_order, float eta_0,
                    float eta_1, float eta_2, float alpha_0, float alpha_1,
                    float alpha_2, float beta, float energy, int64_t n,
                    void* stream) {
    return drift_impl<float>(dt, dE, solver, t_rev, length_ratio, alpha_order,
                             eta_0, eta_1, eta_2, alpha_0, alpha_1, alpha_2,
                             beta, energy, n, stream);
}

int blond_histogram_f64(const double* dt, double* out, double cl, double cr,
                        int S, int64_t n, void* stream) {
    return histogram_impl<double>(dt, out, cl, cr, S, n, stream);
}
int blond_histogram_f32(const float* dt, float* out, float cl, float cr, int S,
                        int64_t n, void* stream) {
    return histogram_impl<float>(dt, out, cl, cr, S, n, stream);
}
int blond_smooth_histogram_f64(const double* dt, double* out, double cl,
                               double cr, int S, int64_t n, void* stream) {
    return smooth_histogram_impl<double>(dt, out, cl, cr, S, n, stream);
}
int blond_smooth_histogram_f32(const float* dt, float* out, float cl, float cr,
                               int S, int64_t n, void* stream) {
    return smooth_histogram_impl<float>(dt, out, cl, cr, S, n, stream);
}

int blond_linear_interp_kick_f64(const double* dt, double* dE, const double* V,
                                 const double* bc, double charge, int S,
                                 int64_t n, double acc, void* stream) {
    return lik_impl<double>(dt, dE, V, bc, charge, S, n, acc, stream);
}
int blond_linear_interp_kick_f32(const float* dt, float* dE, const float* V,
                                 const float* bc, float charge, int S,
                                 int64_t n, float acc, void* stream) {
    return lik_impl<float>(dt, dE, V, bc, charge, S, n, acc, stream);
}

int blond_fast_resonator_f64(double* re, double* im, const double* f,
                             const double* R, const double* Q,
                             const double* fr, int nr, int64_t nf,
                             void* stream) {
    BB_CHECK_ARG(nr >= 0 && nf >= 0, "fast_resonator: negative size");
    if (nr == 0 || nf <= 1) return BLOND_OK;
    BB_CHECK_ARG(re && im && f && R && Q && fr, "fast_resonator: null pointer");
    const int grid = particle_grid(nf, 256, 4);
    fast_resonator_kernel<<<grid, 256, 0, as_stream(stream)>>>(re, im, f, R, Q, fr,
                                                               nr, nf);
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

}  // extern "C"
