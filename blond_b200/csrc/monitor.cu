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

}  // extern "C"
