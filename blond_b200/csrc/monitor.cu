// Beam statistics on the device (Beam.statistics, beam/beam.py:430-458):
// over the particles whose id is non-zero, the mean and standard deviation
// (numpy's, ddof = 0) of dt and dE, the sums of squares, and the rms
// emittance pi sigma_dE sigma_dt.  One pass: every thread accumulates the
// count and the sums of (x - shift) and (x - shift)^2, shift being the
// previous call's mean (so the variance does not cancel: (mean - shift) is
// a small multiple of sigma), and the raw sums of squares; blocks write
// partials, the block that takes the last ticket (no waiting) combines them
// in block order and writes the 8 results.  Nothing is copied to the host:
// a monitor keeps one row per turn on the device.
#include "common.cuh"

namespace bb {
namespace {

constexpr int kStatThreads = 256;
constexpr int kStatVals = 7;  // count, S1 dt, S2 dt, S1 dE, S2 dE, sumsq dt, sumsq dE

template <typename T>
__global__ void __launch_bounds__(kStatThreads)
stats_kernel(const T* __restrict__ dt, const T* __restrict__ dE,
             const int64_t* __restrict__ id, int64_t n, double* __restrict__ stats,
             double* __restrict__ part, int* __restrict__ ticket) {
    // shift: the previous means (stats[1], stats[3]); NaN or inf -> 0
    double sdt = stats[1], sdE = stats[3];
    if (!isfinite(sdt)) sdt = 0.0;
    if (!isfinite(sdE)) sdE = 0.0;
    double v[kStatVals] = {0, 0, 0, 0, 0, 0, 0};
    // four elements per iteration, all loads issued before the arithmetic
    const int64_t G = (int64_t)gridDim.x * kStatThreads;
    for (int64_t i0 = blockIdx.x * (int64_t)kStatThreads + threadIdx.x; i0 < n; i0 += 4 * G) {
        T x[4], y[4];
        bool keep[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t i = i0 + u * G;
            keep[u] = i < n;
            x[u] = keep[u] ? dt[i] : T(0);
            y[u] = keep[u] ? dE[i] : T(0);
            if (id && keep[u]) keep[u] = id[i] != 0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            if (!keep[u]) continue;
            const double xd = (double)x[u], yd = (double)y[u];
            const double a = xd - sdt, b = yd - sdE;
            v[0] += 1.0;
            v[1] += a;
            v[2] += a * a;
            v[3] += b;
            v[4] += b * b;
            v[5] += xd * xd;
            v[6] += yd * yd;
        }
    }
    __shared__ double sh[kStatThreads / 32][kStatVals];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kStatVals; ++q) {
        double s = v[q];
        for (int d = 16; d > 0; d >>= 1) s += __shfl_down_sync(0xffffffffu, s, d);
        if (lane == 0) sh[warp][q] = s;
    }
    __syncthreads();
    if (threadIdx.x < kStatVals) {
        double s = 0.0;
        for (int w = 0; w < kStatThreads / 32; ++w) s += sh[w][threadIdx.x];
        part[(size_t)blockIdx.x * kStatVals + threadIdx.x] = s;
        __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1) == (int)gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the last block combines the partials: thread k sums blocks k, k + 256,
    // ..., then a fixed tree over the threads (the same order every call)
    double t[kStatVals] = {0, 0, 0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < (int)gridDim.x; b += kStatThreads)
#pragma unroll
        for (int q = 0; q < kStatVals; ++q) t[q] += part[(size_t)b * kStatVals + q];
#pragma unroll
    for (int q = 0; q < kStatVals; ++q) {
        double x = t[q];
        for (int d = 16; d > 0; d >>= 1) x += __shfl_down_sync(0xffffffffu, x, d);
        if (lane == 0) sh[warp][q] = x;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
#pragma unroll
    for (int q = 0; q < kStatVals; ++q) {
        double x = 0.0;
        for (int w = 0; w < kStatThreads / 32; ++w) x += sh[w][q];
        t[q] = x;
    }
    *ticket = 0;
    const double cnt = t[0];
    const double m1 = t[1] / cnt, m3 = t[3] / cnt;
    const double var_dt = fmax(t[2] / cnt - m1 * m1, 0.0);
    const double var_dE = fmax(t[4] / cnt - m3 * m3, 0.0);
    const double sig_dt = sqrt(var_dt), sig_dE = sqrt(var_dE);
    stats[0] = cnt;
    stats[1] = sdt + m1;
    stats[2] = sig_dt;
    stats[3] = sdE + m3;
    stats[4] = sig_dE;
    stats[5] = M_PI * sig_dE * sig_dt;
    stats[6] = t[5];
    stats[7] = t[6];
}

template <typename T>
int stats_impl(const T* dt, const T* dE, const int64_t* id, int64_t n, double* stats,
               double* scratch, int* ticket, void* stream) {
    clear_error();
    BB_CHECK_ARG(dt && dE && stats && scratch && ticket, "beam_statistics: null pointer");
    BB_CHECK_SIZE(n >= 1, "beam_statistics: n = %lld (>= 1 required)", (long long)n);
    BB_CHECK_ARG(aligned(dt, sizeof(T)) && aligned(dE, sizeof(T)) && aligned(stats, 8) &&
                     aligned(scratch, 8) && aligned(ticket, 4) && (!id || aligned(id, 8)),
                 "beam_statistics: misaligned array");
    const DeviceInfo& d = device_info();
    int64_t grid = (n + kStatThreads - 1) / kStatThreads;
    grid = grid < (int64_t)d.sm_count * 8 ? grid : (int64_t)d.sm_count * 8;
    if (grid > BLOND_STATS_MAX_BLOCKS) grid = BLOND_STATS_MAX_BLOCKS;
    stats_kernel<T><<<(int)grid, kStatThreads, 0, as_stream(stream)>>>(dt, dE, id, n, stats,
                                                                      scratch, ticket);
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

// ------------------------------------------------------------ cut limits
// CutOptions.set_cuts without given cuts (beam/profile.py:185-195):
//   n_sigma <= 0 (None): cut_left = min - 0.05 (max - min),
//                        cut_right = max + 0.05 (max - min);
//   n_sigma > 0:         cut_left/right = mean -/+ n_sigma sigma / 2
//                        (numpy's mean and population std).
// min and max are exact, so the first form gives the reference's bits; the
// last block evaluates the expressions in the reference's order without
// contraction.  NaN in dt propagates as in numpy.  The mean and std use
// shifted sums (shift = dt[0]), so they agree with numpy's pairwise sums to
// rounding (~1e-16 relative), not bit for bit.
constexpr int kCutThreads = 256;

template <typename T>
__global__ void __launch_bounds__(kCutThreads)
cut_limits_kernel(const T* __restrict__ x, int64_t n, double n_sigma, double* __restrict__ out,
                  double* __restrict__ part, int* __restrict__ ticket) {
    const bool minmax = !(n_sigma > 0);
    const double shift = (double)x[0];
    // minmax: (min, max, nan flag); moments: (S1, S2) of x - shift
    double a = minmax ? INFINITY : 0.0, b = minmax ? -INFINITY : 0.0, nan = 0.0;
    const int64_t G = (int64_t)gridDim.x * kCutThreads;
    for (int64_t i0 = blockIdx.x * (int64_t)kCutThreads + threadIdx.x; i0 < n; i0 += 4 * G) {
        T v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int64_t i = i0 + u * G;
            v[u] = i < n ? x[i] : x[i0];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const double d = (double)v[u];
            if (minmax) {
                if (d != d) nan = 1.0;
                a = fmin(a, d);
                b = fmax(b, d);
            } else if (i0 + u * G < n) {
                const double e = d - shift;
                a += e;
                b += e * e;
            }
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = 16; d > 0; d >>= 1) {
        const double oa = __shfl_down_sync(0xffffffffu, a, d);
        const double ob = __shfl_down_sync(0xffffffffu, b, d);
        nan = fmax(nan, __shfl_down_sync(0xffffffffu, nan, d));
        if (minmax) {
            a = fmin(a, oa);
            b = fmax(b, ob);
        } else {
            a += oa;
            b += ob;
        }
    }
    __shared__ double sh[kCutThreads / 32][3];
    __shared__ bool last;
    if (lane == 0) {
        sh[warp][0] = a;
        sh[warp][1] = b;
        sh[warp][2] = nan;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kCutThreads / 32; ++w) {
            if (minmax) {
                a = fmin(a, sh[w][0]);
                b = fmax(b, sh[w][1]);
            } else {
                a += sh[w][0];
                b += sh[w][1];
            }
            nan = fmax(nan, sh[w][2]);
        }
        part[3 * (size_t)blockIdx.x] = a;
        part[3 * (size_t)blockIdx.x + 1] = b;
        part[3 * (size_t)blockIdx.x + 2] = nan;
        __threadfence();
        last = atomicAdd(ticket, 1) == (int)gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    // the last block combines the partials in block order
    a = minmax ? INFINITY : 0.0;
    b = minmax ? -INFINITY : 0.0;
    nan = 0.0;
    for (int q = 0; q < (int)gridDim.x; ++q) {
        if (minmax) {
            a = fmin(a, part[3 * q]);
            b = fmax(b, part[3 * q + 1]);
        } else {
            a += part[3 * q];
            b += part[3 * q + 1];
        }
        nan = fmax(nan, part[3 * q + 2]);
    }
    *ticket = 0;
    if (minmax) {
        if (nan != 0.0) a = b = NAN;
        // dt_min - 0.05 * (dt_max - dt_min), dt_max + 0.05 * (dt_max - dt_min)
        const double w = __dmul_rn(0.05, __dsub_rn(b, a));
        out[0] = __dsub_rn(a, w);
        out[1] = __dadd_rn(b, w);
    } else {
        const double cnt = (double)n;
        const double m = a / cnt;
        const double mean = shift + m;
        const double sigma = sqrt(fmax(b / cnt - m * m, 0.0));
        // mean - n_sigma * sigma / 2, mean + n_sigma * sigma / 2
        const double h = __ddiv_rn(__dmul_rn(n_sigma, sigma), 2.0);
        out[0] = __dsub_rn(mean, h);
        out[1] = __dadd_rn(mean, h);
    }
}

template <typename T>
int cut_limits_impl(const T* dt, int64_t n, double n_sigma, double* cuts, double* scratch,
                    int* ticket, void* stream) {
    clear_error();
    BB_CHECK_ARG(dt && cuts && scratch && ticket, "cut_limits: null pointer");
    BB_CHECK_SIZE(n >= 1, "cut_limits: n = %lld (>= 1 required)", (long long)n);
    BB_CHECK_ARG(aligned(dt, sizeof(T)) && aligned(cuts, 8) && aligned(scratch, 8) &&
                     aligned(ticket, 4),
                 "cut_limits: misaligned array");
    const DeviceInfo& d = device_info();
    int64_t grid = (n + kCutThreads - 1) / kCutThreads;
    grid = grid < (int64_t)d.sm_count * 8 ? grid : (int64_t)d.sm_count * 8;
    if (grid > BLOND_STATS_MAX_BLOCKS) grid = BLOND_STATS_MAX_BLOCKS;
    cut_limits_kernel<T><<<(int)grid, kCutThreads, 0, as_stream(stream)>>>(
        dt, n, n_sigma, cuts, scratch, ticket);
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

}  // namespace
}  // namespace bb

using namespace bb;

extern "C" {

int blond_beam_statistics_f64(const double* dt, const double* dE, const int64_t* id,
                              int64_t n, double* stats, double* scratch, int* ticket,
                              void* stream) {
    return stats_impl<double>(dt, dE, id, n, stats, scratch, ticket, stream);
}

int blond_beam_statistics_f32(const float* dt, const float* dE, const int64_t* id,
                              int64_t n, double* stats, double* scratch, int* ticket,
                              void* stream) {
    return stats_impl<float>(dt, dE, id, n, stats, scratch, ticket, stream);
}

int blond_cut_limits_f64(const double* dt, int64_t n, double n_sigma, double* cuts,
                         double* scratch, int* ticket, void* stream) {
    return cut_limits_impl<double>(dt, n, n_sigma, cuts, scratch, ticket, stream);
}

int blond_cut_limits_f32(const float* dt, int64_t n, double n_sigma, double* cuts,
                         double* scratch, int* ticket, void* stream) {
    return cut_limits_impl<float>(dt, n, n_sigma, cuts, scratch, ticket, stream);
}

}  // extern "C"
