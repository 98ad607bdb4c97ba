// Differentiable N-turn map and its hand-written adjoint.
//
// One turn t of the forward map, in the reference main loop's order
// (blond/impedances/impedance.py:113-146 then blond/trackers/tracker.py:
// 521-615: induced voltage of the turn-start profile, linear_interp_kick,
// RF kick, drift):
//
//   p_t      = CIC(dt_t)                          profile (counts)
//   V_t      = -s irfft(Z rfft(p_t, n_fft))[:S]   induced voltage, s = q e ratio
//   dE'      = dE_t + q interp(V_t; dt_t) + q sum_j V_j sin(w_j dt_t + phi_j) + acc_t
//   dt_t+1   = dt_t + c_t dE',  dE_t+1 = dE'       simple drift, c_t from turn t+1
//
// CIC is cloud-in-cell deposition on the profile's bin centres
// bc_k = bc_0 + k w: a particle at f = (dt - bc_0)/w gives 1 - u to bin
// floor(f) and u = f - floor(f) to the next, so the profile is continuous
// and piecewise linear in every dt.  (The reference's smooth_histogram,
// blond/cpp_routines/histogram.cpp:75-132, moves a whole particle by two
// bins where it crosses a bin centre, so its profile has no useful
// derivative.)  interp(V; dt) = V_k (1 - u) + V_k+1 u on the same grid is
// the function of linear_interp_kick.cpp:44-62, written without the
// slope/offset cancellation.
//
// The adjoint of one turn, lambda = dL/d(state), runs backwards:
//
//   lambda_dt    += (lambda_p_t+1[k+1] - lambda_p_t+1[k]) / w   at dt_t+1
//   lambda_dE'    = lambda_dE + c_t lambda_dt
//   lambda_dt    += lambda_dE' q (sum_j V_j w_j cos(.) + (V_k+1 - V_k) / w)
//   dL/dV_j,t    += sum_i lambda_dE' q sin(.)
//   dL/dphi_j,t  += sum_i lambda_dE' q V_j cos(.)
//   lambda_V[k]  += lambda_dE' q (1 - u),  lambda_V[k+1] += lambda_dE' q u
//   lambda_dE     = lambda_dE'
//
// followed by lambda_p_t = A^T lambda_V (the same spectral kernel with
// conj(Z): the transpose of a circular convolution is the correlation)
// and the accumulation G += P_t conj(rfft(lambda_V)) from which the host
// forms dL/dZ and, by the chain rule, dL/d(R_s, f_r, Q).  Everything on the
// adjoint side runs in FP64; the forward keeps the engine's FP64 or
// F32P64 (float dE, FP64 phase and drift) arithmetic.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <set>
#include <utility>

#include "../../include/blond_b200.h"
#include "common.cuh"
#include "spectral.cuh"

namespace bb {

constexpr int kAdjThreads = 256;
constexpr int kAdjMaxRf = 4;

struct AdjTurn {
    int64_t n;
    int n_rf;
    const double* V;   // this turn's n_rf amplitudes, frequencies, phases
    const double* om;
    const double* ph;
    double acc, charge, drift_c;
    const double* vind;  // S induced voltages of this turn, or nullptr
    int S;
    double bc0, inv_w;   // bin centres bc0 + k / inv_w
    int smem_hist;       // 1: block-private histograms in shared memory
    int fix_bits;        // fixed-point units per particle: 2^fix_bits
    double fix_scale;    // 2^fix_bits
    int vind_smem;       // 1: a copy of vind in shared memory for the gathers
};

template <int PREC> struct AdjE;
template <> struct AdjE<BLOND_PREC_F64> { using E = double; };
template <> struct AdjE<BLOND_PREC_F32P64> { using E = float; };

__device__ __forceinline__ double adj_reduce_2pi(double x) {
    const double inv2pi = 0.15915494309189533577;
    const double twopi = 6.28318530717958647692;
    return fma(-rint(x * inv2pi), twopi, x);
}

// Cloud-in-cell deposit of a unit weight at dt, in fixed point with 2^b
// units per particle: the weights are w1 = round(u 2^b) and w0 = 2^b - w1,
// accumulated with integer atomics, so every particle deposits exactly one
// unit and the profile does not depend on the order of the atomics (a run
// repeats bit for bit, which finite-difference checks of the map rely
// on).  b = min(52, 62 - ceil(log2(n + 1))) keeps n units below 2^63.
typedef unsigned long long u64;

inline int fixed_bits(int64_t n) {
    int lg = 0;
    while (lg < 63 && (1ull << lg) < (u64)n + 1) ++lg;
    return std::min(52, 62 - lg);
}

// (scale = 2^b: the product is exact, as ldexp's would be; floor(f) is the
// round-down conversion for the f > -1 that get here)
__device__ __forceinline__ void cic_deposit(u64* h, int S, double t, double bc0,
                                            double inv_w, int bits, double scale) {
    const double f = (t - bc0) * inv_w;
    if (!(f > -1.0 && f < (double)S)) return;  // also drops NaN
    const int j = __double2int_rd(f);
    const u64 w1 = (u64)__double2ll_rn((f - (double)j) * scale);
    const u64 w0 = (1ull << bits) - w1;
    if (j >= 0 && w0) atomicAdd(&h[j], w0);
    if (j + 1 < S && w1) atomicAdd(&h[j + 1], w1);
}

__device__ __forceinline__ void zero_shared(u64* h, int S) {
    for (int k = threadIdx.x; k < S; k += blockDim.x) h[k] = 0ull;
}
__device__ __forceinline__ void flush_shared(const u64* h, u64* g, int S) {
    for (int k = threadIdx.x; k < S; k += blockDim.x)
        if (h[k]) atomicAdd(&g[k], h[k]);
}
__device__ __forceinline__ void zero_shared(double* h, int S) {
    for (int k = threadIdx.x; k < S; k += blockDim.x) h[k] = 0.0;
}
__device__ __forceinline__ void flush_shared(const double* h, double* g, int S) {
    for (int k = threadIdx.x; k < S; k += blockDim.x)
        if (h[k] != 0.0) atomicAdd(&g[k], h[k]);
}

// The profile array is accumulated in place as fixed point (its zero bit
// pattern is 0.0) and converted to counts afterwards.
__global__ void fixed_to_counts_kernel(double* p, int S, int bits) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < S; k += gridDim.x * blockDim.x)
        p[k] = ldexp((double)reinterpret_cast<const u64*>(p)[k], -bits);
}

__global__ void __launch_bounds__(kAdjThreads)
adj_deposit_kernel(const double* __restrict__ dt, int64_t n, int S, double bc0, double inv_w,
                   int smem_hist, int bits, u64* __restrict__ prof) {
    extern __shared__ u64 shq[];
    u64* sh = shq;
    u64* h = smem_hist ? sh : prof;
    if (smem_hist) zero_shared(sh, S);
    __syncthreads();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        cic_deposit(h, S, dt[i], bc0, inv_w, bits, ldexp(1.0, bits));
    __syncthreads();
    if (smem_hist) flush_shared(sh, prof, S);
}

// Converts the fixed-point profile to counts in the block that finishes
// last (a counter in global memory, reset by that block), so a turn needs
// no separate conversion launch.  Every block calls it after its own
// deposits; no block waits on another.
__device__ void convert_when_last(u64* prof, int S, int bits, unsigned* done) {
    __shared__ int last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int k = threadIdx.x; k < S; k += blockDim.x)
        reinterpret_cast<double*>(prof)[k] = ldexp((double)__ldcg(prof + k), -bits);
    if (threadIdx.x == 0) *done = 0u;
}

// NRF: the number of RF harmonics, a template parameter so that every
// harmonic's arithmetic is issued only when it exists (a runtime count
// under an unrolled loop to kAdjMaxRf left the unused harmonics' sines
// issued under predicates).
template <int PREC, int NRF>
__global__ void __launch_bounds__(kAdjThreads)
adj_forward_kernel(const AdjTurn T, const double* dt_in, const void* dE_in, double* dt_out,
                   void* dE_out, u64* prof_out, unsigned* done) {
    using E = typename AdjE<PREC>::E;
    // launched with programmatic stream serialization inside the runs: the
    // next grid may launch now; the programme and shared memory are set up
    // before this grid waits for the one before it
    pdl_launch_dependents();
    extern __shared__ u64 shf[];
    __shared__ double sV[kAdjMaxRf], sOm[kAdjMaxRf], sPh[kAdjMaxRf];
    if (threadIdx.x < T.n_rf) {
        sV[threadIdx.x] = T.V[threadIdx.x];
        sOm[threadIdx.x] = T.om[threadIdx.x];
        sPh[threadIdx.x] = T.ph[threadIdx.x];
    }
    const bool dep = prof_out != nullptr;
    const bool hsm = dep && T.smem_hist;
    u64* h = hsm ? shf : prof_out;
    if (hsm) zero_shared(shf, T.S);
    pdl_wait();  // coordinates, induced voltage and counter of the grids before
    const double* vind = T.vind;
    if (vind && T.vind_smem) {
        double* sv = reinterpret_cast<double*>(shf + (hsm ? T.S : 0));
        for (int k = threadIdx.x; k < T.S; k += blockDim.x) sv[k] = T.vind[k];
        vind = sv;
    }
    __syncthreads();
    const E* dEi = static_cast<const E*>(dE_in);
    E* dEo = static_cast<E*>(dE_out);
    const double q = T.charge;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < T.n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double t = dt_in[i];
        E e = dEi[i];
        if (vind) {
            const double f = (t - T.bc0) * T.inv_w;
            if (f >= 0.0 && f < (double)(T.S - 1)) {
                const int k = __double2int_rd(f);
                const double w = f - (double)k;
                e += (E)(q * (vind[k] * (1.0 - w) + vind[k + 1] * w));
            }
        }
        if (PREC == BLOND_PREC_F64) {
            double s = 0.0;
#pragma unroll
            for (int j = 0; j < NRF; ++j) s += sV[j] * sin(fma(sOm[j], t, sPh[j]));
            e += (E)(q * s + T.acc);
        } else {
            // the engine's F32P64 sine: reduction in double, polynomial in float
            float s = 0.0f;
#pragma unroll
            for (int j = 0; j < NRF; ++j) s += (float)sV[j] * rf_sinf(fma(sOm[j], t, sPh[j]));
            e += (E)q * s + (E)T.acc;
        }
        t = t + T.drift_c * (double)e;
        dt_out[i] = t;
        dEo[i] = e;
        if (dep) cic_deposit(h, T.S, t, T.bc0, T.inv_w, T.fix_bits, T.fix_scale);
    }
    if (hsm) {
        __syncthreads();
        flush_shared(shf, prof_out, T.S);
    }
    if (dep && done) convert_when_last(prof_out, T.S, T.fix_bits, done);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// One backward turn (kick = 1), or only the deposit adjoint of a profile
// at dt_next (kick = 0).  Shared memory: lambda_p_next copy, then the
// block's lambda_V accumulator (S doubles each, when smem_hist), then a
// copy of the turn's induced voltage (when vind_smem).
template <int NRF>
__global__ void __launch_bounds__(kAdjThreads)
adj_backward_kernel(const AdjTurn T, int kick, const double* __restrict__ dt,
                    const double* __restrict__ dt_next, const double* __restrict__ lam_p_next,
                    double* __restrict__ lam_dt, double* __restrict__ lam_dE,
                    double* __restrict__ lam_v, double* __restrict__ grad_rf) {
    extern __shared__ double sh[];
    __shared__ double sV[kAdjMaxRf], sOm[kAdjMaxRf], sPh[kAdjMaxRf];
    __shared__ double red[kAdjThreads / 32][2 * kAdjMaxRf];
    const int S = T.S;
    const bool sm = T.smem_hist != 0;
    double* lp = sm ? sh : const_cast<double*>(lam_p_next);
    double* lv = sm ? sh + S : lam_v;
    const double* vind = T.vind;
    pdl_launch_dependents();  // as in adj_forward_kernel
    if (kick && threadIdx.x < T.n_rf) {
        sV[threadIdx.x] = T.V[threadIdx.x];
        sOm[threadIdx.x] = T.om[threadIdx.x];
        sPh[threadIdx.x] = T.ph[threadIdx.x];
    }
    pdl_wait();  // the adjoint and coordinates of the grids before
    if (sm) {
        for (int k = threadIdx.x; k < S; k += blockDim.x) {
            sh[k] = lam_p_next ? lam_p_next[k] : 0.0;
            sh[S + k] = 0.0;
        }
    }
    if (vind && T.vind_smem) {
        double* sv = sh + 2 * S;
        for (int k = threadIdx.x; k < S; k += blockDim.x) sv[k] = T.vind[k];
        vind = sv;
    }
    __syncthreads();
    const double q = T.charge;
    double gv[kAdjMaxRf], gp[kAdjMaxRf];
#pragma unroll
    for (int j = 0; j < kAdjMaxRf; ++j) gv[j] = gp[j] = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < T.n;
         i += (int64_t)gridDim.x * blockDim.x) {
        double ldt = lam_dt[i];
        double ldE = lam_dE[i];
        if (lam_p_next) {
            const double f = (dt_next[i] - T.bc0) * T.inv_w;
            if (f > -1.0 && f < (double)S) {
                const int j = __double2int_rd(f);
                const double a = j >= 0 ? lp[j] : 0.0;
                const double b = j + 1 < S ? lp[j + 1] : 0.0;
                ldt += (b - a) * T.inv_w;
            }
        }
        if (kick) {
            const double t = dt[i];
            const double lE = ldE + T.drift_c * ldt;
            double dg = 0.0;
#pragma unroll
            for (int j = 0; j < NRF; ++j) {
                // sin and cos at the forward's phase, to rounding (the
                // forward map itself keeps CUDA's sin)
                double s, c;
                rf_sincos(fma(sOm[j], t, sPh[j]), &s, &c);
                dg += sV[j] * sOm[j] * c;
                gv[j] += lE * s;
                gp[j] += lE * sV[j] * c;
            }
            dg *= q;
            if (vind) {
                const double f = (t - T.bc0) * T.inv_w;
                if (f >= 0.0 && f < (double)(S - 1)) {
                    const int k = __double2int_rd(f);
                    const double w = f - (double)k;
                    dg += q * (vind[k + 1] - vind[k]) * T.inv_w;
                    atomicAdd(&lv[k], lE * q * (1.0 - w));
                    atomicAdd(&lv[k + 1], lE * q * w);
                }
            }
            ldt += lE * dg;
            ldE = lE;
        }
        lam_dt[i] = ldt;
        lam_dE[i] = ldE;
    }
    if (kick) {
        // programme gradients: warp sums, then one atomic per block and value
        const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
        for (int j = 0; j < NRF; ++j) {
            const double a = warp_sum(gv[j]), b = warp_sum(gp[j]);
            if (lane == 0) {
                red[w][j] = a;
                red[w][kAdjMaxRf + j] = b;
            }
        }
        __syncthreads();
        if (threadIdx.x < 2 * T.n_rf) {
            const int j = threadIdx.x < T.n_rf ? threadIdx.x : kAdjMaxRf + threadIdx.x - T.n_rf;
            double s = 0.0;
            for (int r = 0; r < (int)(blockDim.x >> 5); ++r) s += red[r][j];
            atomicAdd(&grad_rf[threadIdx.x], q * s);
        }
        if (sm) flush_shared(lv, lam_v, S);
    }
}

static int adj_smem_limit() { return (device_info().max_smem_optin - 4096) / 16; }

// Shared memory a block may take for its copy of the induced voltage (with
// the arrays it holds anyway), so that four blocks still fit on an SM.
constexpr size_t kAdjVindSmem = 48 * 1024;

template <typename K>
static int adj_allow_smem(K kernel, bool* done) {
    const DeviceInfo& d = device_info();
    if (!done[d.device & 63]) {
        cudaFuncAttributes fa;
        BB_CUDA(cudaFuncGetAttributes(&fa, kernel));
        BB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     d.max_smem_optin - (int)fa.sharedSizeBytes));
        done[d.device & 63] = true;
    }
    return BLOND_OK;
}

// The same once per kernel and device, for kernels chosen at run time.
template <typename K>
static int adj_allow_smem(K kernel) {
    static std::mutex m;
    static std::set<std::pair<const void*, int>> done;
    const DeviceInfo& d = device_info();
    std::lock_guard<std::mutex> g(m);
    const auto key = std::make_pair(reinterpret_cast<const void*>(kernel), d.device);
    if (done.count(key)) return BLOND_OK;
    cudaFuncAttributes fa;
    BB_CUDA(cudaFuncGetAttributes(&fa, kernel));
    BB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 d.max_smem_optin - (int)fa.sharedSizeBytes));
    done.insert(key);
    return BLOND_OK;
}

// Launch, with programmatic stream serialization when pdl (the turn loops
// of the runs: each grid launches while the one before it finishes).
template <typename... KArgs, typename... Args>
static int adj_launch(void (*k)(KArgs...), int grid, size_t smem, cudaStream_t s, bool pdl,
                      Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kAdjThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    BB_CUDA(cudaLaunchKernelEx(&cfg, k, args...));
    return BLOND_OK;
}

// The kernels for the run-time harmonic count n_rf (0..kAdjMaxRf).
template <int PREC>
static auto adj_forward_for(int n_rf) {
    switch (n_rf) {
        case 0: return adj_forward_kernel<PREC, 0>;
        case 1: return adj_forward_kernel<PREC, 1>;
        case 2: return adj_forward_kernel<PREC, 2>;
        case 3: return adj_forward_kernel<PREC, 3>;
        default: return adj_forward_kernel<PREC, 4>;
    }
}

static auto adj_backward_for(int n_rf) {
    switch (n_rf) {
        case 0: return adj_backward_kernel<0>;
        case 1: return adj_backward_kernel<1>;
        case 2: return adj_backward_kernel<2>;
        case 3: return adj_backward_kernel<3>;
        default: return adj_backward_kernel<4>;
    }
}

// One forward turn.  With a counter (`done`, zero between launches) the
// last block converts the deposited profile to counts; without one a
// second launch does.
static int adj_forward_launch(int precision, const double* dt_in, const void* dE_in,
                              double* dt_out, void* dE_out, int64_t n, int n_rf,
                              const double* voltage, const double* omega_rf,
                              const double* phi_rf, double acc_kick, double charge,
                              double drift_coeff, const double* induced_voltage,
                              int n_slices, double bin_center0, double inv_bin_width,
                              double* profile_out, unsigned* done, void* stream,
                              bool pdl = false) {
    BB_CHECK_ARG(precision == BLOND_PREC_F64 || precision == BLOND_PREC_F32P64,
                 "adjoint_forward_turn: unknown precision %d", precision);
    BB_CHECK_SIZE(n_rf >= 0 && n_rf <= kAdjMaxRf, "adjoint_forward_turn: n_rf=%d not in "
                  "[0, %d]", n_rf, kAdjMaxRf);
    BB_CHECK_ARG(n >= 0 && n_slices >= 2, "adjoint_forward_turn: bad size");
    BB_CHECK_ARG((n == 0 || (dt_in && dE_in && dt_out && dE_out)) &&
                     (n_rf == 0 || (voltage && omega_rf && phi_rf)),
                 "adjoint_forward_turn: null pointer");
    if (n == 0) return BLOND_OK;
    AdjTurn T = {};
    T.n = n;
    T.n_rf = n_rf;
    T.V = voltage;
    T.om = omega_rf;
    T.ph = phi_rf;
    T.acc = acc_kick;
    T.charge = charge;
    T.drift_c = drift_coeff;
    T.vind = induced_voltage;
    T.S = n_slices;
    T.bc0 = bin_center0;
    T.inv_w = inv_bin_width;
    T.smem_hist = n_slices <= adj_smem_limit() ? 1 : 0;
    T.fix_bits = fixed_bits(n);
    T.fix_scale = ldexp(1.0, T.fix_bits);
    const size_t hist = profile_out && T.smem_hist ? sizeof(u64) * n_slices : 0;
    T.vind_smem = induced_voltage && hist + sizeof(double) * n_slices <= kAdjVindSmem;
    const size_t smem = hist + (T.vind_smem ? sizeof(double) * n_slices : 0);
    const int grid = particle_grid(n, kAdjThreads, 4);
    cudaStream_t s = as_stream(stream);
    u64* prof = reinterpret_cast<u64*>(profile_out);
    int rc;
    const auto k = precision == BLOND_PREC_F64 ? adj_forward_for<BLOND_PREC_F64>(n_rf)
                                               : adj_forward_for<BLOND_PREC_F32P64>(n_rf);
    if ((rc = adj_allow_smem(k))) return rc;
    if ((rc = adj_launch(k, grid, smem, s, pdl, T, dt_in, dE_in, dt_out, dE_out, prof, done)))
        return rc;
    if (profile_out && !done) {
        fixed_to_counts_kernel<<<(n_slices + 255) / 256, 256, 0, s>>>(profile_out, n_slices,
                                                                      T.fix_bits);
        BB_LAUNCH_CHECK();
    }
    return BLOND_OK;
}

// One backward turn (blond_adjoint_backward_turn), with programmatic stream
// serialization when pdl.
static int adj_backward_launch(const double* dt, const double* dt_next, int64_t n,
                                double* lam_dt, double* lam_dE, const double* lam_p_next,
                                int kick, int n_rf, const double* voltage,
                                const double* omega_rf, const double* phi_rf, double charge,
                                double drift_coeff, const double* induced_voltage,
                                int n_slices, double bin_center0, double inv_bin_width,
                                double* lam_v, double* grad_rf, void* stream,
                                bool pdl = false) {
    BB_CHECK_SIZE(n_rf >= 0 && n_rf <= kAdjMaxRf, "adjoint_backward_turn: n_rf=%d not in "
                  "[0, %d]", n_rf, kAdjMaxRf);
    BB_CHECK_ARG(n >= 0 && n_slices >= 2, "adjoint_backward_turn: bad size");
    BB_CHECK_ARG(n == 0 || (lam_dt && lam_dE), "adjoint_backward_turn: null adjoint");
    BB_CHECK_ARG(!lam_p_next || dt_next, "adjoint_backward_turn: lam_p_next needs dt_next");
    BB_CHECK_ARG(!kick || ((n == 0 || dt) && grad_rf && (!induced_voltage || lam_v) &&
                           (n_rf == 0 || (voltage && omega_rf && phi_rf))),
                 "adjoint_backward_turn: null pointer");
    if (n == 0) return BLOND_OK;
    AdjTurn T = {};
    T.n = n;
    T.n_rf = n_rf;
    T.V = voltage;
    T.om = omega_rf;
    T.ph = phi_rf;
    T.charge = charge;
    T.drift_c = drift_coeff;
    T.vind = kick ? induced_voltage : nullptr;
    T.S = n_slices;
    T.bc0 = bin_center0;
    T.inv_w = inv_bin_width;
    T.smem_hist = n_slices <= adj_smem_limit() ? 1 : 0;
    T.vind_smem = T.vind && T.smem_hist && 3 * sizeof(double) * n_slices <= kAdjVindSmem;
    int rc;
    const auto k = adj_backward_for(kick ? n_rf : 0);
    if ((rc = adj_allow_smem(k))) return rc;
    const size_t smem = T.smem_hist ? (T.vind_smem ? 3 : 2) * sizeof(double) * n_slices : 0;
    const int grid = particle_grid(n, kAdjThreads, 4);
    return adj_launch(k, grid, smem, as_stream(stream), pdl, T, kick, dt, dt_next, lam_p_next,
                      lam_dt, lam_dE, lam_v, grad_rf);
}

}  // namespace bb

using namespace bb;

extern "C" {

int blond_adjoint_deposit(const double* dt, int64_t n, int n_slices, double bin_center0,
                          double inv_bin_width, double* profile, void* stream) {
    BB_CHECK_ARG(n >= 0 && n_slices >= 1, "adjoint_deposit: bad size");
    BB_CHECK_ARG(profile && (n == 0 || dt), "adjoint_deposit: null pointer");
    if (n == 0) return BLOND_OK;
    static bool done[64] = {false};
    int rc;
    if ((rc = adj_allow_smem(adj_deposit_kernel, done))) return rc;
    const int sm = n_slices <= adj_smem_limit() ? 1 : 0;
    const int grid = particle_grid(n, kAdjThreads, 4);
    cudaStream_t s = as_stream(stream);
    adj_deposit_kernel<<<grid, kAdjThreads, sm ? sizeof(u64) * n_slices : 0, s>>>(
        dt, n, n_slices, bin_center0, inv_bin_width, sm, fixed_bits(n),
        reinterpret_cast<u64*>(profile));
    BB_LAUNCH_CHECK();
    fixed_to_counts_kernel<<<(n_slices + 255) / 256, 256, 0, s>>>(profile, n_slices,
                                                                  fixed_bits(n));
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

int blond_adjoint_forward_turn(int precision, const double* dt_in, const void* dE_in,
                               double* dt_out, void* dE_out, int64_t n, int n_rf,
                               const double* voltage, const double* omega_rf,
                               const double* phi_rf, double acc_kick, double charge,
                               double drift_coeff, const double* induced_voltage,
                               int n_slices, double bin_center0, double inv_bin_width,
                               double* profile_out, void* stream) {
    return adj_forward_launch(precision, dt_in, dE_in, dt_out, dE_out, n, n_rf, voltage,
                              omega_rf, phi_rf, acc_kick, charge, drift_coeff,
                              induced_voltage, n_slices, bin_center0, inv_bin_width,
                              profile_out, nullptr, stream);
}

int blond_adjoint_backward_turn(const double* dt, const double* dt_next, int64_t n,
                                double* lam_dt, double* lam_dE, const double* lam_p_next,
                                int kick, int n_rf, const double* voltage,
                                const double* omega_rf, const double* phi_rf, double charge,
                                double drift_coeff, const double* induced_voltage,
                                int n_slices, double bin_center0, double inv_bin_width,
                                double* lam_v, double* grad_rf, void* stream) {
    return adj_backward_launch(dt, dt_next, n, lam_dt, lam_dE, lam_p_next, kick, n_rf, voltage,
                               omega_rf, phi_rf, charge, drift_coeff, induced_voltage, n_slices,
                               bin_center0, inv_bin_width, lam_v, grad_rf, stream);
}

int blond_adjoint_spectral(int mode, const double* x, int n_slices, const double* impedance,
                           int64_t n_fft, double scale, double* y, double* spectrum,
                           double* accum, void* stream) {
    BB_CHECK_ARG(mode == 0 || mode == 1, "adjoint_spectral: mode must be 0 or 1");
    BB_CHECK_ARG(x && impedance && y && n_slices >= 1, "adjoint_spectral: bad argument");
    BB_CHECK_ARG(mode == 0 || (spectrum && accum), "adjoint_spectral: mode 1 needs the "
                 "stored spectrum and the accumulator");
    SpecParams P = {};
    if (!make_spec_plan(n_fft, P.p)) {
        set_error("adjoint_spectral: n_fft=%lld is not an even 5-smooth length <= %lld",
                  (long long)n_fft, (long long)kMaxClusterFFT);
        return BLOND_ERR_UNSUPPORTED;
    }
    P.mode = SPEC_FORWARD | SPEC_MULTIPLY | SPEC_INVERSE;
    P.in_f64 = x;
    P.n_in = n_slices;
    P.H = reinterpret_cast<const double2*>(impedance);
    P.out = y;
    P.n_out = n_slices < n_fft ? n_slices : n_fft;
    P.out_scale = -scale / (double)P.p.M;
    if (mode == 0 && spectrum) {
        P.mode |= SPEC_OUT_SPECTRUM;
        P.spec_out = reinterpret_cast<double2*>(spectrum);
    }
    if (mode == 1) {
        P.mode |= SPEC_ACCUM;
        P.acc_a = reinterpret_cast<const double2*>(spectrum);
        P.acc_g = reinterpret_cast<double2*>(accum);
    }
    return launch_spectral(P, as_stream(stream));
}

}  // extern "C"

namespace bb {

// The induced-voltage transform of the turn loops below: one plan and one
// twiddle table for the whole run (the per-turn entry point builds the plan
// on the host and the twiddles in the kernel at every call).
struct AdjSpectral {
    SpecPlan plan = {};
    double2* tw = nullptr;
    ~AdjSpectral() {
        if (tw) cudaFree(tw);
    }
    int init(int64_t n_fft) {
        if (!make_spec_plan(n_fft, plan)) {
            set_error("adjoint run: n_fft=%lld is not an even 5-smooth length <= %lld",
                      (long long)n_fft, (long long)kMaxClusterFFT);
            return BLOND_ERR_UNSUPPORTED;
        }
        int rc;
        if ((rc = prepare_spectral())) return rc;
        return make_spec_twiddles(plan, &tw);
    }
    // the same transform as blond_adjoint_spectral(mode, ...)
    int run(int mode, const double* x, int S, const double* H, double scale, double* y,
            double* spectrum, double* accum, cudaStream_t s) const {
        SpecParams P = {};
        P.p = plan;
        P.twg = tw;
        P.pdl = 1;  // inside the turn loops of the runs
        P.mode = SPEC_FORWARD | SPEC_MULTIPLY | SPEC_INVERSE;
        P.in_f64 = x;
        P.n_in = S;
        P.H = reinterpret_cast<const double2*>(H);
        P.out = y;
        P.n_out = S < plan.N ? S : plan.N;
        P.out_scale = -scale / (double)plan.M;
        if (mode == 0 && spectrum) {
            P.mode |= SPEC_OUT_SPECTRUM;
            P.spec_out = reinterpret_cast<double2*>(spectrum);
        }
        if (mode == 1) {
            P.mode |= SPEC_ACCUM;
            P.acc_a = reinterpret_cast<const double2*>(spectrum);
            P.acc_g = reinterpret_cast<double2*>(accum);
        }
        return launch_spectral(P, s);
    }
};

// A zeroed device counter for the forward kernel's last-block conversion,
// owned by one run.
struct AdjCounter {
    unsigned* p = nullptr;
    ~AdjCounter() {
        if (p) cudaFree(p);
    }
    int init(cudaStream_t s) {
        BB_CUDA(cudaMalloc(&p, sizeof(unsigned)));
        BB_CUDA(cudaMemsetAsync(p, 0, sizeof(unsigned), s));
        return BLOND_OK;
    }
};

}  // namespace bb

extern "C" {

int blond_adjoint_forward_run(int precision, double* dt, void* dE, int64_t n, int n_rf,
                              int64_t n_turns, const double* voltage, const double* omega_rf,
                              const double* phi_rf, const double* acc_kick,
                              const double* drift_coeff, double charge,
                              const double* impedance, int64_t n_fft, double scale,
                              double* induced_voltage, double* spectrum, double* profile,
                              int n_slices, double bin_center0, double inv_bin_width,
                              int checkpoint_every, double* ckpt_dt, void* ckpt_dE,
                              void* stream) {
    BB_CHECK_ARG(precision == BLOND_PREC_F64 || precision == BLOND_PREC_F32P64,
                 "adjoint_forward_run: precision must be F64 or F32P64");
    BB_CHECK_ARG(n >= 1 && n_turns >= 1 && n_slices >= 2 && checkpoint_every >= 1,
                 "adjoint_forward_run: bad size");
    BB_CHECK_ARG(dt && dE && voltage && omega_rf && phi_rf && acc_kick && drift_coeff &&
                     profile && ckpt_dt && ckpt_dE,
                 "adjoint_forward_run: null pointer");
    BB_CHECK_ARG(!impedance || (induced_voltage && spectrum),
                 "adjoint_forward_run: an impedance needs the induced-voltage and spectrum "
                 "arrays");
    cudaStream_t s = as_stream(stream);
    const size_t esz = precision == BLOND_PREC_F64 ? sizeof(double) : sizeof(float);
    const int64_t M1 = n_fft / 2 + 1;
    AdjSpectral sp;
    AdjCounter done;
    int rc;
    if (impedance && (rc = sp.init(n_fft))) return rc;
    if ((rc = done.init(s))) return rc;
    if ((rc = blond_adjoint_deposit(dt, n, n_slices, bin_center0, inv_bin_width, profile,
                                    stream)))
        return rc;
    for (int64_t t = 0; t < n_turns; ++t) {
        if (t % checkpoint_every == 0) {
            const int64_t seg = t / checkpoint_every;
            BB_CUDA(cudaMemcpyAsync(ckpt_dt + seg * n, dt, sizeof(double) * n,
                                    cudaMemcpyDeviceToDevice, s));
            BB_CUDA(cudaMemcpyAsync(static_cast<char*>(ckpt_dE) + (size_t)seg * n * esz, dE,
                                    esz * n, cudaMemcpyDeviceToDevice, s));
        }
        double* vind = impedance ? induced_voltage + t * n_slices : nullptr;
        if (impedance &&
            (rc = sp.run(0, profile + t * n_slices, n_slices, impedance, scale, vind,
                         spectrum + t * M1 * 2, nullptr, s)))
            return rc;
        if ((rc = adj_forward_launch(
                 precision, dt, dE, dt, dE, n, n_rf, voltage + t * n_rf, omega_rf + t * n_rf,
                 phi_rf + t * n_rf, acc_kick[t], charge, drift_coeff[t], vind, n_slices,
                 bin_center0, inv_bin_width, profile + (t + 1) * n_slices, done.p, stream,
                 true)))
            return rc;
    }
    return BLOND_OK;
}

int blond_adjoint_backward_run(int precision, int64_t n, int n_rf, int64_t n_turns,
                               const double* voltage, const double* omega_rf,
                               const double* phi_rf, const double* acc_kick,
                               const double* drift_coeff, double charge,
                               const double* impedance_conj, int64_t n_fft, double scale,
                               const double* induced_voltage, const double* spectrum,
                               int n_slices, double bin_center0, double inv_bin_width,
                               int checkpoint_every, const double* ckpt_dt,
                               const void* ckpt_dE, double* states, void* dE_work,
                               double* lam_dt, double* lam_dE, const double* lam_p_final,
                               double* lam_v, double* lam_pt, double* grad_rf,
                               double* spectrum_accum, void* stream) {
    BB_CHECK_ARG(precision == BLOND_PREC_F64 || precision == BLOND_PREC_F32P64,
                 "adjoint_backward_run: precision must be F64 or F32P64");
    BB_CHECK_ARG(n >= 1 && n_turns >= 1 && n_slices >= 2 && checkpoint_every >= 1,
                 "adjoint_backward_run: bad size");
    BB_CHECK_ARG(voltage && omega_rf && phi_rf && acc_kick && drift_coeff && ckpt_dt &&
                     ckpt_dE && states && dE_work && lam_dt && lam_dE && grad_rf,
                 "adjoint_backward_run: null pointer");
    BB_CHECK_ARG(!impedance_conj || (induced_voltage && spectrum && lam_v && lam_pt &&
                                     spectrum_accum),
                 "adjoint_backward_run: an impedance needs the stored induced voltages and "
                 "spectra and the adjoint arrays");
    cudaStream_t s = as_stream(stream);
    const size_t esz = precision == BLOND_PREC_F64 ? sizeof(double) : sizeof(float);
    const int64_t M1 = n_fft / 2 + 1;
    const int64_t K = checkpoint_every;
    const int64_t nseg = (n_turns + K - 1) / K;
    const bool has_z = impedance_conj != nullptr;
    AdjSpectral sp;
    int rc;
    if (has_z && (rc = sp.init(n_fft))) return rc;
    const double* lam_p = lam_p_final;
    for (int64_t seg = nseg - 1; seg >= 0; --seg) {
        const int64_t a = seg * K, b = std::min(n_turns, (seg + 1) * K);
        // the segment's turn-start coordinates, recomputed from its checkpoint
        BB_CUDA(cudaMemcpyAsync(states, ckpt_dt + seg * n, sizeof(double) * n,
                                cudaMemcpyDeviceToDevice, s));
        BB_CUDA(cudaMemcpyAsync(dE_work, static_cast<const char*>(ckpt_dE) + (size_t)seg * n * esz,
                                esz * n, cudaMemcpyDeviceToDevice, s));
        for (int64_t t = a; t < b; ++t) {
            if ((rc = adj_forward_launch(
                     precision, states + (t - a) * n, dE_work, states + (t - a + 1) * n,
                     dE_work, n, n_rf, voltage + t * n_rf, omega_rf + t * n_rf,
                     phi_rf + t * n_rf, acc_kick[t], charge, drift_coeff[t],
                     has_z ? induced_voltage + t * n_slices : nullptr, n_slices, bin_center0,
                     inv_bin_width, nullptr, nullptr, stream, true)))
                return rc;
        }
        for (int64_t t = b - 1; t >= a; --t) {
            if ((rc = adj_backward_launch(
                     states + (t - a) * n, states + (t - a + 1) * n, n, lam_dt, lam_dE, lam_p, 1,
                     n_rf, voltage + t * n_rf, omega_rf + t * n_rf, phi_rf + t * n_rf, charge,
                     drift_coeff[t], has_z ? induced_voltage + t * n_slices : nullptr,
                     n_slices, bin_center0, inv_bin_width,
                     has_z ? lam_v + t * n_slices : nullptr, grad_rf + t * 2 * n_rf, stream,
                     true)))
                return rc;
            if (has_z) {
                if ((rc = sp.run(1, lam_v + t * n_slices, n_slices, impedance_conj, scale,
                                 lam_pt + t * n_slices, const_cast<double*>(spectrum) + t * M1 * 2,
                                 spectrum_accum, s)))
                    return rc;
                lam_p = lam_pt + t * n_slices;
            } else {
                lam_p = nullptr;
            }
        }
    }
    // the turn-0 profile is a deposit of the initial dt
    if (lam_p)
        return blond_adjoint_backward_turn(nullptr, ckpt_dt, n, lam_dt, lam_dE, lam_p, 0, n_rf,
                                           nullptr, nullptr, nullptr, charge, 0.0, nullptr,
                                           n_slices, bin_center0, inv_bin_width, nullptr,
                                           nullptr, stream);
    return BLOND_OK;
}

}  // extern "C"
