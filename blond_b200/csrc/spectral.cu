// Host side of the cluster FFT (plan, launch) and the C ABI for rfft,
// irfft and the one-turn induced voltage; plus a direct-DFT path for the
// lengths the cluster transform does not take (odd, or prime factors > 5).
#define BB_SPECTRAL_KERNELS
#include "spectral.cuh"

#include <vector>

namespace bb {

// Radix passes of a length-L transform: as few as possible (each pass is a
// block barrier and a shared-memory round trip), radix 8 first.
static void radix_schedule(int L, int* r, int& n) {
    n = 0;
    while (L % 8 == 0) { r[n++] = 8; L /= 8; }
    while (L % 4 == 0) { r[n++] = 4; L /= 4; }
    while (L % 2 == 0) { r[n++] = 2; L /= 2; }
    while (L % 3 == 0) { r[n++] = 3; L /= 3; }
    while (L % 5 == 0) { r[n++] = 5; L /= 5; }
}

static bool smooth5(int64_t x) {
    if (x < 1) return false;
    for (int f : {2, 3, 5})
        while (x % f == 0) x /= f;
    return x == 1;
}

bool make_spec_plan(int64_t N, SpecPlan& plan, int max_cluster) {
    if (N < 2 || (N & 1) || N > kMaxClusterFFT) return false;
    const int M = (int)(N / 2);
    if (!smooth5(M)) return false;
    // Pick M1 | M (M1 <= M2) maximising the cluster size C (a power of two
    // dividing both factors, with at least 64 points per CTA), then the
    // most square split.
    int best_m1 = 1, best_c = 1;
    double best_score = -1.0;
    for (int m1 = 1; (int64_t)m1 * m1 <= M; ++m1) {
        if (M % m1) continue;
        const int m2 = M / m1;
        int cc = 1;
        while (cc * 2 <= max_cluster && m1 % (cc * 2) == 0 && m2 % (cc * 2) == 0 &&
               M / (cc * 2) >= 64)
            cc *= 2;
        const double score = cc * 1e6 + (double)m1 / (double)m2;
        if (score > best_score) {
            best_score = score;
            best_m1 = m1;
            best_c = cc;
        }
    }
    plan.N = (int)N;
    plan.M = M;
    plan.M1 = best_m1;
    plan.M2 = M / best_m1;
    plan.C = best_c;
    plan.Bc = plan.M2 / plan.C;
    plan.Br = plan.M1 / plan.C;
    radix_schedule(plan.M1, plan.r1, plan.n1);
    radix_schedule(plan.M2, plan.r2, plan.n2);
    plan.L = 1;
    while ((int64_t)plan.L * plan.L < M) plan.L *= 2;
    // fewest cluster barriers (three buffers) and staged impedance when the
    // shared memory allows, else fall back step by step
    const int budget = device_info().max_smem_optin;
    const int options[4][2] = {{3, 1}, {3, 0}, {2, 1}, {2, 0}};
    for (const auto& o : options) {
        plan.nbuf = o[0];
        plan.prefetch = o[1];
        plan.smem = spec_layout(plan).total;
        if (plan.smem <= budget) break;
    }
    return true;
}

int prepare_spectral() {
    static bool attr_done[64] = {false};
    const DeviceInfo& d = device_info();
    if (!attr_done[d.device & 63]) {
        BB_CUDA(cudaFuncSetAttribute(spectral_kernel<false>,
                                     cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        BB_CUDA(cudaFuncSetAttribute(spectral_kernel<false>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     d.max_smem_optin));
        BB_CUDA(cudaFuncSetAttribute(spectral_kernel<true>,
                                     cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
        BB_CUDA(cudaFuncSetAttribute(spectral_kernel<true>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     d.max_smem_optin));
        attr_done[d.device & 63] = true;
    }
    return BLOND_OK;
}

template <bool FB>
static int launch_spectral_t(const SpecParams& P, const typename SpecLoopArg<FB>::type& L,
                             cudaStream_t stream) {
    const DeviceInfo& d = device_info();
    if (P.p.smem > d.max_smem_optin) {
        set_error("spectral: %d B of shared memory per CTA exceeds %d", P.p.smem,
                  d.max_smem_optin);
        return BLOND_ERR_SIZE;
    }
    int rc = prepare_spectral();
    if (rc) return rc;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(P.p.C * (P.batch > 0 ? P.batch : 1), 1, 1);
    cfg.blockDim = dim3(kSpecThreads, 1, 1);
    cfg.dynamicSmemBytes = P.p.smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = P.p.C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = P.pdl ? 2 : 1;
    BB_CUDA(cudaLaunchKernelEx(&cfg, spectral_kernel<FB>, P, L));
    return BLOND_OK;
}

int launch_spectral(const SpecParams& P, cudaStream_t stream) {
    return launch_spectral_t<false>(P, SpecNoLoop{}, stream);
}

int launch_spectral_loop(const SpecParams& P, const SpecLoop& L, cudaStream_t stream) {
    if (P.batch > 0) {
        set_error("spectral: the beam-phase loop runs with a single profile");
        return BLOND_ERR_UNSUPPORTED;
    }
    return launch_spectral_t<true>(P, L, stream);
}

__global__ void twiddle_table_kernel(const SpecPlan p, double2* out) {
    const SpecLayout lay = spec_layout(p);
    double2* base = out;
    auto at = [&](int off) { return base + (off - lay.tw1) / 16; };
    fill_twiddles(p, at(lay.tw1), at(lay.tw2), at(lay.tam), at(lay.tbm), at(lay.tan_),
                  at(lay.tbn), threadIdx.x, blockDim.x);
}

int make_spec_twiddles(const SpecPlan& plan, double2** out) {
    const SpecLayout lay = spec_layout(plan);
    const size_t bytes = (size_t)(lay.hk - lay.tw1);
    *out = nullptr;
    BB_CUDA(cudaMalloc(out, bytes));
    twiddle_table_kernel<<<1, 512>>>(plan, *out);
    BB_LAUNCH_CHECK();
    BB_CUDA(cudaDeviceSynchronize());
    return BLOND_OK;
}

// ---------------------------------------------------------------- direct DFT
// Single-CTA O(N^2) transforms for short lengths the cluster plan rejects.
// Twiddles are indexed (k n mod N) from a shared table.
constexpr int kDirectThreads = 512;

__global__ void __launch_bounds__(kDirectThreads)
direct_rfft_kernel(const double* __restrict__ x, int64_t n_x, int N,
                   double2* __restrict__ out, const double2* __restrict__ H,
                   double2* __restrict__ keep_spectrum) {
    extern __shared__ double2 tw[];
    for (int q = threadIdx.x; q < N; q += blockDim.x) tw[q] = twiddle<false>(q, N);
    __syncthreads();
    const int nk = N / 2 + 1;
    const int nx = (int)(n_x < N ? n_x : N);
    for (int k = threadIdx.x; k < nk; k += blockDim.x) {
        double re = 0.0, im = 0.0;
        int e = 0;
        for (int n = 0; n < nx; ++n) {
            const double2 w = tw[e];
            re += x[n] * w.x;
            im += x[n] * w.y;
            e += k;
            if (e >= N) e -= N;
        }
        double2 X = make_double2(re, im);
        if (keep_spectrum) keep_spectrum[k] = X;
        if (H) X = cmul(X, H[k]);
        out[k] = X;
    }
}

// irfft of length N from spectrum Y[0..n_y-1] (missing entries are zero,
// imaginary parts of Y[0] and Y[N/2] ignored), y[n] = scale * (...).
__global__ void __launch_bounds__(kDirectThreads)
direct_irfft_kernel(const double2* __restrict__ Y, int64_t n_y, int N,
                    double* __restrict__ y, int64_t n_out, double scale) {
    extern __shared__ double2 tw[];
    for (int q = threadIdx.x; q < N; q += blockDim.x) tw[q] = twiddle<true>(q, N);
    __syncthreads();
    const int half = N / 2;
    const int kmax = (int)((int64_t)(N - 1) / 2 < n_y - 1 ? (N - 1) / 2 : n_y - 1);
    for (int n = threadIdx.x; n < n_out && n < N; n += blockDim.x) {
        double acc = n_y > 0 ? Y[0].x : 0.0;
        int e = n;
        for (int k = 1; k <= kmax; ++k) {
            const double2 w = tw[e];
            acc += 2.0 * (Y[k].x * w.x - Y[k].y * w.y);
            e += n;
            if (e >= N) e -= N;
        }
        if ((N & 1) == 0 && half < n_y) acc += Y[half].x * ((n & 1) ? -1.0 : 1.0);
        y[n] = acc * scale;
    }
}

static int direct_smem(int N) { return (int)sizeof(double2) * N; }

static int set_direct_attrs() {
    static bool done[64] = {false};
    const DeviceInfo& d = device_info();
    if (!done[d.device & 63]) {
        BB_CUDA(cudaFuncSetAttribute(direct_rfft_kernel,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     direct_smem((int)kMaxDirectDFT)));
        BB_CUDA(cudaFuncSetAttribute(direct_irfft_kernel,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     direct_smem((int)kMaxDirectDFT)));
        done[d.device & 63] = true;
    }
    return BLOND_OK;
}

}  // namespace bb

using namespace bb;

extern "C" {

int blond_rfft_f64(const double* x, int64_t n_x, int64_t n_fft, double* spectrum,
                   void* stream) {
    BB_CHECK_ARG(n_x >= 0 && n_fft >= 1, "rfft: bad length (n_x=%lld, n_fft=%lld)",
                 (long long)n_x, (long long)n_fft);
    BB_CHECK_ARG(spectrum && (n_x == 0 || x), "rfft: null pointer");
    cudaStream_t s = as_stream(stream);
    SpecParams P = {};
    if (make_spec_plan(n_fft, P.p)) {
        P.mode = SPEC_FORWARD | SPEC_OUT_SPECTRUM;
        P.in_f64 = x;
        P.n_in = n_x;
        P.spec_out = reinterpret_cast<double2*>(spectrum);
        return launch_spectral(P, s);
    }
    if (n_fft > kMaxDirectDFT) {
        set_error("rfft: n_fft=%lld is neither an even 5-smooth length <= %lld nor "
                  "<= %lld", (long long)n_fft, (long long)kMaxClusterFFT,
                  (long long)kMaxDirectDFT);
        return BLOND_ERR_UNSUPPORTED;
    }
    int rc = set_direct_attrs();
    if (rc) return rc;
    direct_rfft_kernel<<<1, kDirectThreads, direct_smem((int)n_fft), s>>>(
        x, n_x, (int)n_fft, reinterpret_cast<double2*>(spectrum), nullptr, nullptr);
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

int blond_irfft_f64(const double* spectrum, int64_t n_fft, double* y,
                    int64_t n_out, void* stream) {
    BB_CHECK_ARG(n_fft >= 1 && n_out >= 0, "irfft: bad length");
    BB_CHECK_ARG(spectrum && (n_out == 0 || y), "irfft: null pointer");
    if (n_out > n_fft) n_out = n_fft;
    cudaStream_t s = as_stream(stream);
    SpecParams P = {};
    if (make_spec_plan(n_fft, P.p)) {
        P.mode = SPEC_IN_SPECTRUM | SPEC_INVERSE;
        P.spec_in = reinterpret_cast<const double2*>(spectrum);
        P.n_spec_in = n_fft / 2 + 1;
        P.out = y;
        P.n_out = n_out;
        P.out_scale = 1.0 / (double)P.p.M;
        return launch_spectral(P, s);
    }
    if (n_fft > kMaxDirectDFT) {
        set_error("irfft: n_fft=%lld unsupported", (long long)n_fft);
        return BLOND_ERR_UNSUPPORTED;
    }
    int rc = set_direct_attrs();
    if (rc) return rc;
    direct_irfft_kernel<<<1, kDirectThreads, direct_smem((int)n_fft), s>>>(
        reinterpret_cast<const double2*>(spectrum), n_fft / 2 + 1, (int)n_fft, y, n_out,
        1.0 / (double)n_fft);
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

int blond_induced_voltage_f64(const double* profile, int n_slices,
                              const double* impedance, int64_t n_fft,
                              double scale, double* v_out, int64_t n_out,
                              void* stream) {
    BB_CHECK_ARG(n_slices >= 1 && n_fft >= 1 && n_out >= 0,
                 "induced_voltage: bad length");
    BB_CHECK_ARG(profile && impedance && (n_out == 0 || v_out),
                 "induced_voltage: null pointer");
    cudaStream_t s = as_stream(stream);
    SpecParams P = {};
    if (make_spec_plan(n_fft, P.p)) {
        P.mode = SPEC_FORWARD | SPEC_MULTIPLY | SPEC_INVERSE;
        P.in_f64 = profile;
        P.n_in = n_slices;
        P.H = reinterpret_cast<const double2*>(impedance);
        P.out = v_out;
        P.n_out = n_out < n_fft ? n_out : n_fft;
        P.out_scale = -scale / (double)P.p.M;
        return launch_spectral(P, s);
    }
    set_error("induced_voltage: n_fft=%lld is not an even 5-smooth length <= %lld; "
              "use blond_rfft_f64/blond_irfft_f64", (long long)n_fft,
              (long long)kMaxClusterFFT);
    return BLOND_ERR_UNSUPPORTED;
}

}  // extern "C"
