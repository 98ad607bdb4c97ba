// Time-domain wake kernels.
//
// 1. The analytic resonator convolution of InducedVoltageResonator
//    (impedances/impedance.py:1042-1335; the arithmetic is
//    resonator_induced_voltage_1_turn, utils/butils_wrap_python.py:656-790).
//    The reference evaluates, for every time t_j and every bin k,
//        F_r(D) = (2 cos(a D) + sin(a D)/Qt) exp(-b D) H(D) - sign(D),
//        D = t_j - bc_k,
//        V_j = scale * sum_r R/(2 w Q) sum_k kappa_k (F_r(D_j,k+1) - F_r(D_j,k)),
//    an n_time x n_slices matrix per resonator.  With p = -b + i a and
//    c = 2 - i/Qt, F_r(D) = Re[c e^{pD}] - 1 for D > 0 and 1 for D <= 0, so
//    the sum over the bins below t_j factors through e^{p t_j}.  Writing
//    m = #{k : bc_k < t_j} and i = m - 1 (bin centres increasing),
//        sum_k kappa_k (F_{k+1} - F_k)
//            = Re[c e^{p (t_j - bc_i)} (J_i - kappa_i)] + 2 kappa_i,
//        J_0 = 0,  J_i = e^{p h_i} J_{i-1} - kappa_{i-1} expm1(p h_i),
//        h_i = bc_i - bc_{i-1},  kappa_{S-1} = 0,
//    and the sum is 0 when m = 0.  Every exponential has a non-positive
//    real part, so nothing overflows where the reference's exp(-b D) for
//    D < 0 does (it then multiplies inf by 0 and returns NaN).  The work is
//    O(n_slices) per resonator for the recurrence (resonator_scan_kernel, a
//    block-wide scan of the affine maps J -> A J + B) plus O(log n_slices)
//    per time point (resonator_eval_kernel) instead of O(n_slices) per time
//    point.
//
// 2. numpy.interp (bm.interp, utils/bmath_backends.py:373) for the
//    multi-turn-wake memory shift of _InducedVoltage.shift_trev_time
//    (impedance.py:533-550).
#include "common.cuh"

namespace bb {
namespace {

constexpr int kScanThreads = 512;
constexpr int kScanCache = 4;  // elements a scan thread keeps in registers
constexpr int kEvalThreads = 256;

struct cplx {
    double re, im;
};

// Per-resonator constants, passed by value (impedance.py:1218-1220):
// qt = Q sqrt(1 - 1/(4 Q^2)), a = w qt / Q, b = w / (2 Q), coef = R / (2 w Q).
// a_pi = a / pi feeds sincospi, whose argument reduction is exact and cheap
// at any magnitude (a t reaches 1e7 rad over a long multi-turn memory).
struct ResonatorParams {
    int n;
    double qt[BLOND_MAX_RESONATORS], a[BLOND_MAX_RESONATORS], b[BLOND_MAX_RESONATORS],
        coef[BLOND_MAX_RESONATORS], a_pi[BLOND_MAX_RESONATORS];
};
__device__ __forceinline__ cplx cmul(cplx a, cplx b) {
    return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__device__ __forceinline__ cplx cadd(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
// e^{x + i pi y}
__device__ __forceinline__ cplx cexp_pi(double x, double y) {
    double s, c;
    sincospi(y, &s, &c);
    const double m = exp(x);
    return {m * c, m * s};
}
// e^{x + iy} - 1 without cancellation for small |x + iy|, from one sincos
// of y/2 (s, c) and expm1(x) = m:
// Re = m cos y - 2 s^2 with cos y = 1 - 2 s^2, Im = (m + 1) 2 s c.
__device__ __forceinline__ cplx cexpm1(double x, double y) {
    double s, c;
    sincos(0.5 * y, &s, &c);
    const double m = expm1(x);
    const double s2 = 2.0 * s * s;
    return {m * (1.0 - s2) - s2, (m + 1.0) * (2.0 * s * c)};
}
__device__ __forceinline__ cplx shfl_up(cplx v, int d) {
    return {__shfl_up_sync(0xffffffffu, v.re, d), __shfl_up_sync(0xffffffffu, v.im, d)};
}

// (A, B) := (A, B) o (Ae, Be): the affine map J -> Ae J + Be first, then
// J -> A J + B.
__device__ __forceinline__ void compose(cplx& A, cplx& B, cplx Ae, cplx Be) {
    const cplx nA = cmul(A, Ae);
    const cplx nB = cadd(cmul(A, Be), B);
    A = nA;
    B = nB;
}

// kappa_k, as the reference forms it: diff(profile) / diff(bin_centers) /
// (beam_n_macroparticles * bin_size), with kappa_{S-1} = 0 past the end.
__device__ __forceinline__ double kappa_at(const double* prof, const double* bc, int S,
                                           int k, double nb) {
    if (k >= S - 1) return 0.0;
    return div_rn(div_rn(sub_rn(prof[k + 1], prof[k]), sub_rn(bc[k + 1], bc[k])), nb);
}

// Element i of the recurrence, J_i = lam J_{i-1} + add.
struct Elem {
    cplx lam, add;
};
__device__ __forceinline__ Elem scan_elem(const double* prof, const double* bc, int S, int i,
                                          double nb, double a, double b) {
    const double h = bc[i] - bc[i - 1];
    const cplx em1 = cexpm1(-b * h, a * h);
    const double kp = kappa_at(prof, bc, S, i - 1, nb);
    return {{em1.re + 1.0, em1.im}, {-kp * em1.re, -kp * em1.im}};
}
__device__ __forceinline__ cplx apply(const Elem& e, cplx J) {
    return {e.lam.re * J.re - e.lam.im * J.im + e.add.re,
            e.lam.re * J.im + e.lam.im * J.re + e.add.im};
}

// One block per resonator: J_i for i in [0, S) into J[r * S + i], and
// (block 0) kappa_k for k in [0, S) into kappa.  Each thread takes a
// contiguous segment of elements; the first kScanCache stay in registers
// between the two passes, the rest are recomputed.
__global__ void __launch_bounds__(kScanThreads, 1)
resonator_scan_kernel(const double* __restrict__ prof, const double* __restrict__ bc,
                      int S, double nb, ResonatorParams rp, double* __restrict__ kappa,
                      double2* __restrict__ J) {
    constexpr int kWarps = kScanThreads / 32;
    const int r = blockIdx.x;
    const int t = threadIdx.x;
    const int lane = t & 31, warp = t >> 5;
    const double a = rp.a[r], b = rp.b[r];
    const int n_el = S - 1;  // elements i = 1 .. S-1
    const int per = (n_el + kScanThreads - 1) / kScanThreads;
    const int lo = 1 + t * per;
    const int hi = min(S, lo + per);

    if (r == 0)
        for (int k = t; k < S; k += kScanThreads) kappa[k] = kappa_at(prof, bc, S, k, nb);

    // pass 1: this thread's segment as one affine map J -> A J + B
    Elem cache[kScanCache];
    cplx A = {1.0, 0.0}, B = {0.0, 0.0};
#pragma unroll
    for (int q = 0; q < kScanCache; ++q) {
        const int i = lo + q;
        if (i < hi) {
            cache[q] = scan_elem(prof, bc, S, i, nb, a, b);
            A = cmul(cache[q].lam, A);
            B = apply(cache[q], B);
        }
    }
    for (int i = lo + kScanCache; i < hi; ++i) {
        const Elem e = scan_elem(prof, bc, S, i, nb, a, b);
        A = cmul(e.lam, A);
        B = apply(e, B);
    }

    // inclusive warp scan, then over warp totals
    __shared__ cplx sA[kWarps], sB[kWarps];
    for (int d = 1; d < 32; d <<= 1) {
        const cplx Ae = shfl_up(A, d), Be = shfl_up(B, d);
        if (lane >= d) compose(A, B, Ae, Be);
    }
    if (lane == 31) {
        sA[warp] = A;
        sB[warp] = B;
    }
    __syncthreads();
    if (warp == 0) {
        cplx wA = {1.0, 0.0}, wB = {0.0, 0.0};
        if (lane < kWarps) {
            wA = sA[lane];
            wB = sB[lane];
        }
        for (int d = 1; d < kWarps; d <<= 1) {
            const cplx Ae = shfl_up(wA, d), Be = shfl_up(wB, d);
            if (lane >= d) compose(wA, wB, Ae, Be);
        }
        if (lane < kWarps) {
            sA[lane] = wA;
            sB[lane] = wB;
        }
    }
    __syncthreads();
    // exclusive prefix of this thread = (inclusive of lane-1) o (warps before)
    cplx eA = shfl_up(A, 1), eB = shfl_up(B, 1);
    if (lane == 0) {
        eA = {1.0, 0.0};
        eB = {0.0, 0.0};
    }
    if (warp > 0) compose(eA, eB, sA[warp - 1], sB[warp - 1]);

    // pass 2: replay the segment from the carried-in J_{lo-1} = eB
    cplx Jc = eB;
    double2* Jr = J + (size_t)r * S;
    if (t == 0) Jr[0] = make_double2(0.0, 0.0);
#pragma unroll
    for (int q = 0; q < kScanCache; ++q) {
        const int i = lo + q;
        if (i < hi) {
            Jc = apply(cache[q], Jc);
            Jr[i] = make_double2(Jc.re, Jc.im);
        }
    }
    for (int i = lo + kScanCache; i < hi; ++i) {
        Jc = apply(scan_elem(prof, bc, S, i, nb, a, b), Jc);
        Jr[i] = make_double2(Jc.re, Jc.im);
    }
}

// #{k : bc_k < x} over increasing bc.
__device__ __forceinline__ int count_below_search(const double* __restrict__ bc, int S,
                                                  double x) {
    int lo = 0, hi = S;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (bc[mid] < x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// The same from the evenly spaced estimate (x - bc_0) / mean spacing,
// corrected by a short walk; the binary search when the walk is long
// (uneven bins).  Exact for any increasing bc.
__device__ __forceinline__ int count_below(const double* __restrict__ bc, int S, double x,
                                           double bc0, double inv_h) {
    double f = ceil((x - bc0) * inv_h);
    f = fmin(fmax(f, 0.0), (double)S);
    int m = (int)f;
    for (int it = 0; it < 4; ++it) {
        if (m < S && bc[m] < x) {
            ++m;
        } else if (m > 0 && !(bc[m - 1] < x)) {
            --m;
        } else {
            return m;
        }
    }
    return count_below_search(bc, S, x);
}

// G = 2^log_g lanes per output point (G >= n_resonators up to 32), lane
// q of a group taking modes q, q + G, ...; the group sums its modes with
// shuffles.  MTW = false: out[j] = V_j for j < n_time.  MTW = true
// (InducedVoltageResonator.induced_voltage_mtw, impedance.py:1317-1335):
// out is the new memory of n_out points,
//     out[j] = mem_in[j + shift] (0 past its end) + V_j (j < n_time),
// the reference's append-zeros / drop-one-window / add in one pass.
template <bool MTW>
__global__ void __launch_bounds__(kEvalThreads)
resonator_eval_kernel(const double* __restrict__ time_array, int64_t n_time,
                      const double* __restrict__ bc, int S,
                      const double* __restrict__ kappa, const double2* __restrict__ J,
                      ResonatorParams rp, int log_g, double scale, double* __restrict__ out,
                      int64_t n_out, const double* __restrict__ mem_in, int64_t shift,
                      double* __restrict__ per_resonator) {
    const double bc0 = bc[0];
    const double inv_h = S > 1 ? (double)(S - 1) / (bc[S - 1] - bc0) : 0.0;
    const int G = 1 << log_g;
    const int q = threadIdx.x & (G - 1);
    const int64_t total = n_out << log_g;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    // every lane of a warp runs the same iterations (the shuffles need them)
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < total; base += stride) {
        const int64_t g = base + threadIdx.x;
        const int64_t j = g >> log_g;
        const bool active = g < total;
        double sum = 0.0;
        bool nan_t = false;
        if (active && j < n_time) {
            const double tj = time_array[j];
            if (tj != tj) {  // NaN time: the reference's sum is NaN too
                nan_t = true;
                sum = tj;
                if (per_resonator)
                    for (int r = q; r < rp.n; r += G) per_resonator[(size_t)r * n_time + j] = tj;
            } else {
                const int m = count_below(bc, S, tj, bc0, inv_h);
                const int i = m - 1;
                const double kp = m > 0 ? kappa[i] : 0.0;
                const double d = m > 0 ? tj - bc[i] : 0.0;
                for (int r = q; r < rp.n; r += G) {
                    double v = 0.0;
                    if (m > 0) {
                        const double2 Ji = J[(size_t)r * S + i];
                        const cplx E = cexp_pi(-rp.b[r] * d, rp.a_pi[r] * d);
                        const cplx O = cmul(E, {Ji.x - kp, Ji.y});
                        v = (2.0 * O.re + O.im / rp.qt[r]) + 2.0 * kp;
                    }
                    const double tr = rp.coef[r] * v;
                    if (per_resonator) per_resonator[(size_t)r * n_time + j] = tr;
                    sum += tr;
                }
            }
        }
        for (int w = 1; w < G; w <<= 1) sum += __shfl_xor_sync(0xffffffffu, sum, w);
        if (!active || q != 0) continue;
        const double v_total = j < n_time ? (nan_t ? sum : sum * scale) : 0.0;
        if (MTW) {
            const int64_t src = j + shift;
            const double old = src < n_out ? mem_in[src] : 0.0;
            out[j] = j < n_time ? old + v_total : old;
        } else {
            out[j] = v_total;
        }
    }
}

// numpy.interp: left / right outside [xp_0, xp_{m-1}], fp_{m-1} at the last
// point, fp_j where x equals xp_j, else slope (x - xp_j) + fp_j with the
// slope (fp_{j+1} - fp_j) / (xp_{j+1} - xp_j), retried from the right end
// of the interval if that is NaN.  No FMA contraction: numpy's C loop rounds
// the product and the sum separately.
__global__ void __launch_bounds__(kEvalThreads)
interp_kernel(const double* __restrict__ x, int64_t n, double x_shift,
              const double* __restrict__ xp, const double* __restrict__ fp, int m,
              double left, double right, int flags, double* __restrict__ out) {
    const double lval = (flags & 1) ? left : fp[0];
    const double rval = (flags & 2) ? right : fp[m - 1];
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n;
         q += (int64_t)gridDim.x * blockDim.x) {
        const double xv = add_rn(x[q], x_shift);
        double res;
        if (xv != xv) {
            res = xv;
        } else if (xv < xp[0]) {
            res = lval;
        } else if (xv > xp[m - 1]) {
            res = rval;
        } else {
            // largest j with xp_j <= xv
            int lo = 0, hi = m;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (xp[mid] <= xv)
                    lo = mid;
                else
                    hi = mid;
            }
            const int j = lo;
            if (j == m - 1 || xp[j] == xv) {
                res = fp[j];
            } else {
                const double slope = div_rn(sub_rn(fp[j + 1], fp[j]), sub_rn(xp[j + 1], xp[j]));
                res = add_rn(mul_rn(slope, sub_rn(xv, xp[j])), fp[j]);
                if (res != res) {
                    res = add_rn(mul_rn(slope, sub_rn(xv, xp[j + 1])), fp[j + 1]);
                    if (res != res && fp[j] == fp[j + 1]) res = fp[j];
                }
            }
        }
        out[q] = res;
    }
}

int eval_grid(int64_t n) {
    const DeviceInfo& d = device_info();
    int64_t need = (n + kEvalThreads - 1) / kEvalThreads;
    int64_t cap = (int64_t)d.sm_count * 8;
    if (need < 1) need = 1;
    return (int)(need < cap ? need : cap);
}

bool overlaps(const void* a, size_t na, const void* b, size_t nb) {
    const uintptr_t pa = reinterpret_cast<uintptr_t>(a), pb = reinterpret_cast<uintptr_t>(b);
    return pa < pb + nb && pb < pa + na;
}

}  // namespace
}  // namespace bb

using namespace bb;

extern "C" {

int64_t blond_resonator_workspace_bytes(int n_slices, int n_resonators) {
    if (n_slices < 1 || n_resonators < 1) return 0;
    return (int64_t)n_resonators * n_slices * 16 + (int64_t)n_slices * 8;
}

static int resonator_launch(const double* n_macroparticles, const double* bin_centers,
                            int n_slices, double bin_size, double beam_n_macroparticles,
                            const double* time_array, int64_t n_time, const double* R_S,
                            const double* omega_R, const double* Q, int n_resonators,
                            double scale, double* out, int64_t n_out, const double* mem_in,
                            int64_t shift, double* tmp_matrix, void* workspace,
                            int64_t workspace_bytes, void* stream) {
    BB_CHECK_ARG(n_macroparticles && bin_centers && time_array && R_S && omega_R && Q && out &&
                     workspace,
                 "resonator_induced_voltage: null pointer");
    BB_CHECK_SIZE(n_slices >= 1 && n_slices <= (1 << 24),
                  "resonator_induced_voltage: n_slices %d outside [1, 2^24]", n_slices);
    BB_CHECK_SIZE(n_time >= 0, "resonator_induced_voltage: negative n_time");
    BB_CHECK_SIZE(n_resonators >= 1 && n_resonators <= BLOND_MAX_RESONATORS,
                  "resonator_induced_voltage: %d resonators, supported 1..%d", n_resonators,
                  BLOND_MAX_RESONATORS);
    BB_CHECK_ARG(workspace_bytes >= blond_resonator_workspace_bytes(n_slices, n_resonators),
                 "resonator_induced_voltage: workspace of %lld bytes, need %lld",
                 (long long)workspace_bytes,
                 (long long)blond_resonator_workspace_bytes(n_slices, n_resonators));
    BB_CHECK_ARG(aligned(workspace, 16) && aligned(n_macroparticles, 8) &&
                     aligned(bin_centers, 8) && aligned(time_array, 8) && aligned(out, 8) &&
                     (!tmp_matrix || aligned(tmp_matrix, 8)) && (!mem_in || aligned(mem_in, 8)),
                 "resonator_induced_voltage: misaligned array");
    const size_t no = (size_t)n_out * 8, nt = (size_t)n_time * 8;
    const size_t nw = (size_t)workspace_bytes;
    BB_CHECK_ARG(!overlaps(out, no, workspace, nw) &&
                     (!mem_in || !overlaps(out, no, mem_in, no)) &&
                     (!tmp_matrix || (!overlaps(tmp_matrix, nt * n_resonators, workspace, nw) &&
                                      !overlaps(tmp_matrix, nt * n_resonators, out, no))),
                 "resonator_induced_voltage: an output overlaps an input or the workspace");

    // Resonator constants in the reference's operation order
    // (impedance.py:1218-1220, butils_wrap_python.py:777-781).
    ResonatorParams rp;
    rp.n = n_resonators;
    for (int r = 0; r < n_resonators; ++r) {
        BB_CHECK_ARG(Q[r] >= 0.5 && omega_R[r] > 0.0,
                     "resonator_induced_voltage: resonator %d has Q = %g, omega_R = %g "
                     "(Q >= 0.5 and omega_R > 0 required)",
                     r, Q[r], omega_R[r]);
        const double qt = Q[r] * sqrt(1.0 - 1.0 / (4.0 * (Q[r] * Q[r])));
        rp.qt[r] = qt;
        rp.a[r] = omega_R[r] * qt / Q[r];
        rp.a_pi[r] = rp.a[r] / M_PI;
        rp.b[r] = omega_R[r] / (2.0 * Q[r]);
        rp.coef[r] = R_S[r] / (2.0 * omega_R[r] * Q[r]);
    }
    const double nb = beam_n_macroparticles * bin_size;
    double2* J = reinterpret_cast<double2*>(workspace);
    double* kappa = reinterpret_cast<double*>(J + (size_t)n_resonators * n_slices);
    cudaStream_t s = as_stream(stream);
    resonator_scan_kernel<<<n_resonators, kScanThreads, 0, s>>>(
        n_macroparticles, bin_centers, n_slices, nb, rp, kappa, J);
    BB_LAUNCH_CHECK();
    if (n_out > 0) {
        int log_g = 0;
        while ((1 << log_g) < n_resonators && log_g < 5) ++log_g;
        const int grid = eval_grid(n_out << log_g);
        if (mem_in)
            resonator_eval_kernel<true><<<grid, kEvalThreads, 0, s>>>(
                time_array, n_time, bin_centers, n_slices, kappa, J, rp, log_g, scale, out,
                n_out, mem_in, shift, tmp_matrix);
        else
            resonator_eval_kernel<false><<<grid, kEvalThreads, 0, s>>>(
                time_array, n_time, bin_centers, n_slices, kappa, J, rp, log_g, scale, out,
                n_out, nullptr, 0, tmp_matrix);
        BB_LAUNCH_CHECK();
    }
    return BLOND_OK;
}

int blond_resonator_induced_voltage_f64(
    const double* n_macroparticles, const double* bin_centers, int n_slices,
    double bin_size, double beam_n_macroparticles, const double* time_array,
    int64_t n_time, const double* R_S, const double* omega_R, const double* Q,
    int n_resonators, double scale, double* induced_voltage, double* tmp_matrix,
    void* workspace, int64_t workspace_bytes, void* stream) {
    clear_error();
    return resonator_launch(n_macroparticles, bin_centers, n_slices, bin_size,
                            beam_n_macroparticles, time_array, n_time, R_S, omega_R, Q,
                            n_resonators, scale, induced_voltage, n_time, nullptr, 0,
                            tmp_matrix, workspace, workspace_bytes, stream);
}

int blond_resonator_mtw_f64(
    const double* n_macroparticles, const double* bin_centers, int n_slices,
    double bin_size, double beam_n_macroparticles, const double* time_array,
    int64_t n_time, const double* R_S, const double* omega_R, const double* Q,
    int n_resonators, double scale, const double* memory_in, double* memory_out,
    int64_t n_memory, int64_t shift, double* tmp_matrix, void* workspace,
    int64_t workspace_bytes, void* stream) {
    clear_error();
    BB_CHECK_ARG(memory_in, "resonator_mtw: null memory_in");
    BB_CHECK_SIZE(n_memory >= n_time && shift >= 0,
                  "resonator_mtw: memory of %lld points, n_time %lld, shift %lld "
                  "(n_memory >= n_time and shift >= 0 required)",
                  (long long)n_memory, (long long)n_time, (long long)shift);
    return resonator_launch(n_macroparticles, bin_centers, n_slices, bin_size,
                            beam_n_macroparticles, time_array, n_time, R_S, omega_R, Q,
                            n_resonators, scale, memory_out, n_memory, memory_in, shift,
                            tmp_matrix, workspace, workspace_bytes, stream);
}

int blond_interp_f64(const double* x, int64_t n, double x_shift, const double* xp,
                     const double* fp, int m, double left, double right, int flags,
                     double* out, void* stream) {
    clear_error();
    BB_CHECK_ARG(x && xp && fp && out, "interp: null pointer");
    BB_CHECK_SIZE(n >= 0 && m >= 1, "interp: n = %lld, m = %d (m >= 1 required)",
                  (long long)n, m);
    BB_CHECK_ARG(!overlaps(out, (size_t)n * 8, fp, (size_t)m * 8) &&
                     !overlaps(out, (size_t)n * 8, xp, (size_t)m * 8),
                 "interp: out overlaps xp or fp");
    BB_CHECK_ARG(aligned(x, 8) && aligned(xp, 8) && aligned(fp, 8) && aligned(out, 8),
                 "interp: misaligned array");
    if (n == 0) return BLOND_OK;
    interp_kernel<<<eval_grid(n), kEvalThreads, 0, as_stream(stream)>>>(
        x, n, x_shift, xp, fp, m, left, right, flags, out);
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

}  // extern "C"
