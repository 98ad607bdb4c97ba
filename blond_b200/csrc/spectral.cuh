// Cluster-resident real FFT convolution used for the induced voltage.
//
// The reference computes V = -q e ratio * irfft(Z * rfft(profile, n_fft))
// with numpy's pocketfft (blond/impedances/impedance.py:457-489) -- a
// latency-bound O(n log n) step between two HBM-bound particle passes.  Here
// the whole chain runs in ONE launch of one thread-block cluster (up to 16
// CTAs): the real input of length N = 2M is packed into M complex points,
// transformed by a four-step FFT (M = M1 x M2) whose transpose goes through
// distributed shared memory, post-processed into the N/2+1 real-input
// spectrum, multiplied by the impedance, pre-processed back and inverse
// transformed the same way.  No global scratch; the profile is read once
// and the voltage (plus the particle kernel's interpolation table) written
// once.
//
// In-CTA transforms are batched mixed-radix (2/3/4/5) Stockham passes
// (the autosort formulation of Govindaraju et al., "High performance
// discrete Fourier transforms on graphics processors", SC 2008) over an
// interleaved batch layout element(b, i) = buf[i * B + b].  Twiddles come
// from sincospi() in double precision.
#pragma once

#include <cooperative_groups.h>

#include "common.cuh"

namespace bb {

namespace cg = cooperative_groups;

constexpr int kSpecThreads = 256;
constexpr int kMaxPasses = 24;
constexpr int kMaxCluster = 16;
constexpr int64_t kMaxClusterFFT = 131072;  // real length N
constexpr int64_t kMaxDirectDFT = 4096;

struct SpecPlan {
    int N;        // real transform length (even)
    int M;        // N / 2 complex points
    int M1, M2;   // M = M1 * M2
    int C;        // CTAs in the cluster; divides M1 and M2
    int Bc, Br;   // M2 / C columns and M1 / C rows per CTA
    int n1, n2;   // radix passes for M1 and M2
    int r1[kMaxPasses], r2[kMaxPasses];
    int smem;     // dynamic shared memory per CTA, bytes
};

// Bits of SpecParams::mode
enum : int {
    SPEC_FORWARD = 1,     // input is real: pack, forward transform
    SPEC_INVERSE = 2,     // run the inverse transform and write real output
    SPEC_OUT_SPECTRUM = 4,// write the N/2+1 spectrum of the real input
    SPEC_IN_SPECTRUM = 8, // input is an N/2+1 spectrum (irfft only)
    SPEC_MULTIPLY = 16,   // multiply the spectrum by H before inverting
};

struct SpecParams {
    SpecPlan p;
    int mode;
    // real input (profile): exactly one of in_f64 / in_i32 is set
    const double* in_f64;
    int* in_i32;          // engine histogram; zeroed after it is read
    int64_t n_in;
    double* profile_out;  // engine: converted profile (n_in doubles)
    const double2* spec_in;  // SPEC_IN_SPECTRUM: n_spec_in complex values
    int64_t n_spec_in;
    const double2* H;     // SPEC_MULTIPLY: M + 1 values
    double2* spec_out;    // SPEC_OUT_SPECTRUM: M + 1 values
    double* out;          // SPEC_INVERSE: real output
    int64_t n_out;
    double out_scale;     // applied to the real output
    // engine extras ---------------------------------------------------
    // inductive impedance: out[k] += ind_coeff[turn] * gradient(profile)[k]
    const double* ind_coeff;  // per turn, already includes 1/bin_size
    double ind_dbc;           // bin_centers[1] - bin_centers[0]
    // interpolation table for the particle kernel over the n_out voltages
    void* table;              // nullptr = none
    int table_f32;            // 0: double2 {slope, offset}; 1: float2 {qV, slope}
    double charge, inv_w;     // inv_w = (S-1)/(bc[S-1]-bc[0])
    const double* bc;
    long long* turn;          // device turn counter (read; incremented if bump)
    int bump_turn;
};

// Device code below is compiled only in spectral.cu (which defines
// BB_SPECTRAL_KERNELS); other files see the types and host entry points.
#ifdef BB_SPECTRAL_KERNELS

// ------------------------------------------------------------ complex ops
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ double2 crot(double2 a) {
    return INV ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}
// exp(-2 pi i num / den) (forward) or its conjugate
template <bool INV>
__device__ __forceinline__ double2 twiddle(long long num, long long den) {
    double s, c;
    sincospi(2.0 * (double)num / (double)den, &s, &c);
    return make_double2(c, INV ? s : -s);
}

// ------------------------------------------------------------ radix kernels
template <bool INV>
__device__ __forceinline__ void dft2(double2* v) {
    const double2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
}
template <bool INV>
__device__ __forceinline__ void dft4(double2* v) {
    const double2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
    const double2 s13 = cadd(v[1], v[3]), d13 = crot<INV>(csub(v[1], v[3]));
    v[0] = cadd(s02, s13);
    v[2] = csub(s02, s13);
    v[1] = cadd(d02, d13);
    v[3] = csub(d02, d13);
}
template <bool INV>
__device__ __forceinline__ void dft3(double2* v) {
    const double h = 0.86602540378443864676;  // sin(2 pi / 3)
    const double2 a = v[0], s = cadd(v[1], v[2]), d = csub(v[1], v[2]);
    const double2 m = make_double2(a.x - 0.5 * s.x, a.y - 0.5 * s.y);
    const double2 r = crot<INV>(cscale(d, h));
    v[0] = cadd(a, s);
    v[1] = cadd(m, r);
    v[2] = csub(m, r);
}
template <bool INV>
__device__ __forceinline__ void dft5(double2* v) {
    const double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;
    const double s1 = 0.95105651629515357212, s2 = 0.58778525229247312917;
    const double2 a = v[0];
    const double2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    const double2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    const double2 m1 = make_double2(a.x + c1 * t1.x + c2 * t2.x, a.y + c1 * t1.y + c2 * t2.y);
    const double2 m2 = make_double2(a.x + c2 * t1.x + c1 * t2.x, a.y + c2 * t1.y + c1 * t2.y);
    const double2 r1 = crot<INV>(make_double2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y));
    const double2 r2 = crot<INV>(make_double2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y));
    v[0] = cadd(a, cadd(t1, t2));
    v[1] = cadd(m1, r1);
    v[4] = csub(m1, r1);
    v[2] = cadd(m2, r2);
    v[3] = csub(m2, r2);
}

// One Stockham pass of radix R over B interleaved transforms of length L.
template <bool INV, int R>
__device__ __forceinline__ void stockham_pass(const double2* __restrict__ src,
                                              double2* __restrict__ dst, int L,
                                              int B, int Ns,
                                              const double2* __restrict__ tw) {
    const int LR = L / R;
    const int total = B * LR;
    const int step = L / (Ns * R);
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int b = idx % B;
        const int j = idx / B;
        const int k = j % Ns;
        double2 v[R];
#pragma unroll
        for (int t = 0; t < R; ++t) {
            double2 x = src[(j + t * LR) * B + b];
            if (t > 0 && k > 0) {
                double2 w = tw[t * k * step];
                if (INV) w.y = -w.y;
                x = cmul(x, w);
            }
            v[t] = x;
        }
        if (R == 2) dft2<INV>(v);
        if (R == 3) dft3<INV>(v);
        if (R == 4) dft4<INV>(v);
        if (R == 5) dft5<INV>(v);
        const int d = (j / Ns) * Ns * R + k;
#pragma unroll
        for (int t = 0; t < R; ++t) dst[(d + t * Ns) * B + b] = v[t];
    }
}

// B transforms of length L, interleaved, starting in a[]; returns the buffer
// (a or b) that holds the result.  Ends with __syncthreads().
template <bool INV>
__device__ double2* batch_fft(double2* a, double2* b, int L, int B,
                              const int* radices, int npass,
                              const double2* tw) {
    int Ns = 1;
    for (int p = 0; p < npass; ++p) {
        const int R = radices[p];
        if (R == 4) stockham_pass<INV, 4>(a, b, L, B, Ns, tw);
        else if (R == 2) stockham_pass<INV, 2>(a, b, L, B, Ns, tw);
        else if (R == 3) stockham_pass<INV, 3>(a, b, L, B, Ns, tw);
        else stockham_pass<INV, 5>(a, b, L, B, Ns, tw);
        __syncthreads();
        double2* t = a;
        a = b;
        b = t;
        Ns *= R;
    }
    return a;
}

// ------------------------------------------------------------ the kernel
// One cluster of p.C CTAs.  Column phase: CTA c owns n2 in [c Bc, (c+1) Bc),
// element (n1, n2) at n1 * Bc + n2 - c Bc.  Row phase: CTA c owns k1 in
// [c Br, (c+1) Br), element (k1, k2) at k2 * Br + k1 - c Br.
__global__ void __launch_bounds__(kSpecThreads)
spectral_kernel(const SpecParams P) {
    cg::cluster_group cluster = cg::this_cluster();
    const SpecPlan& p = P.p;
    const int c = (int)cluster.block_rank();
    const int tid = threadIdx.x, nth = blockDim.x;
    extern __shared__ double2 smem[];
    const int per = p.M / p.C;
    double2* buf0 = smem;
    double2* buf1 = smem + per;
    double2* tw1 = smem + 2 * per;     // M1 entries
    double2* tw2 = tw1 + p.M1;         // M2 entries
    const int M = p.M, M1 = p.M1, M2 = p.M2, Bc = p.Bc, Br = p.Br;

    for (int q = tid; q < M1; q += nth) tw1[q] = twiddle<false>(q, M1);
    for (int q = tid; q < M2; q += nth) tw2[q] = twiddle<false>(q, M2);
    const long long turn = P.turn ? *P.turn : 0;

    double2* rows = nullptr;  // row-phase buffer holding Z (forward) / U
    double2* other = nullptr;

    if (P.mode & SPEC_FORWARD) {
        // ---- load: z[m] = x[2m] + i x[2m+1], m = c Bc + b + M2 n1
        const int64_t nlim = P.n_in < (int64_t)p.N ? P.n_in : (int64_t)p.N;
        for (int e = tid; e < per; e += nth) {
            const int b = e % Bc, n1 = e / Bc;
            const int64_t m = (int64_t)c * Bc + b + (int64_t)M2 * n1;
            double x0 = 0.0, x1 = 0.0;
            const int64_t i0 = 2 * m, i1 = 2 * m + 1;
            if (P.in_i32) {
                if (i0 < nlim) { x0 = (double)P.in_i32[i0]; P.in_i32[i0] = 0; }
                if (i1 < nlim) { x1 = (double)P.in_i32[i1]; P.in_i32[i1] = 0; }
                if (P.profile_out) {
                    if (i0 < P.n_in) P.profile_out[i0] = x0;
                    if (i1 < P.n_in) P.profile_out[i1] = x1;
                }
            } else {
                if (i0 < nlim) x0 = P.in_f64[i0];
                if (i1 < nlim) x1 = P.in_f64[i1];
            }
            buf0[n1 * Bc + b] = make_double2(x0, x1);
        }
        // histogram bins beyond the transform length (profile longer than
        // n_fft): converted and cleared but not transformed
        if (P.in_i32 && c == 0) {
            for (int64_t i = (int64_t)p.N + tid; i < P.n_in; i += nth) {
                const double x = (double)P.in_i32[i];
                P.in_i32[i] = 0;
                if (P.profile_out) P.profile_out[i] = x;
            }
        }
        __syncthreads();
        // ---- column transforms (length M1 over n1, Bc of them)
        double2* colres = batch_fft<false>(buf0, buf1, M1, Bc, p.r1, p.n1, tw1);
        double2* colfree = colres == buf0 ? buf1 : buf0;
        cluster.sync();
        // ---- transpose into rows with the four-step twiddle W_M^(n2 k1)
        for (int e = tid; e < Br * M2; e += nth) {
            const int n2 = e % M2, br = e / M2;
            const int k1 = c * Br + br;
            const int owner = n2 / Bc;
            const double2* remote = cluster.map_shared_rank(colres, owner);
            double2 v = remote[k1 * Bc + (n2 - owner * Bc)];
            const long long ex = ((long long)n2 * k1) % M;
            if (ex) v = cmul(v, twiddle<false>(ex, M));
            colfree[n2 * Br + br] = v;
        }
        cluster.sync();
        // ---- row transforms (length M2 over n2, Br of them) -> Z[k1 + M1 k2]
        rows = batch_fft<false>(colfree, colres, M2, Br, p.r2, p.n2, tw2);
        other = rows == colfree ? colres : colfree;
        cluster.sync();
    }

    if (P.mode & (SPEC_OUT_SPECTRUM | SPEC_MULTIPLY | SPEC_IN_SPECTRUM)) {
        if (!rows) {
            rows = buf0;
            other = buf1;
        }
        // ---- spectral step on own k = k1 + M1 k2 with partner M - k
        for (int e = tid; e < per; e += nth) {
            const int br = e % Br, k2 = e / Br;
            const int k1 = c * Br + br;
            const int k = k1 + M1 * k2;
            const int pk = (M - k) % M;
            double2 Yk, Yp;  // Y[k], Y[M-k] (Y[M] when k == 0)
            if (P.mode & SPEC_IN_SPECTRUM) {
                const int64_t kk = k, kp = (k == 0) ? M : (M - k);
                Yk = kk < P.n_spec_in ? P.spec_in[kk] : make_double2(0, 0);
                Yp = kp < P.n_spec_in ? P.spec_in[kp] : make_double2(0, 0);
            } else {
                const int p1 = pk % M1, p2 = pk / M1, owner = p1 / Br;
                const double2* remote = cluster.map_shared_rank(rows, owner);
                const double2 Zk = rows[k2 * Br + br];
                const double2 Zp = remote[p2 * Br + (p1 - owner * Br)];
                if (k == 0) {
                    Yk = make_double2(Zk.x + Zk.y, 0.0);  // X[0]
                    Yp = make_double2(Zk.x - Zk.y, 0.0);  // X[M]
                } else {
                    const double2 E = cscale(cadd(Zk, cconj(Zp)), 0.5);
                    const double2 O = crot<false>(cscale(csub(Zk, cconj(Zp)), 0.5));
                    const double2 wk = twiddle<false>(k, 2LL * M);  // e^{-2 pi i k/N}
                    const double2 wO = cmul(wk, O);
                    Yk = cadd(E, wO);                 // X[k]
                    Yp = cconj(csub(E, wO));          // X[M-k]
                }
                if (P.mode & SPEC_OUT_SPECTRUM) {
                    // every k < M is owned once; X[M] comes from k == 0
                    P.spec_out[k] = Yk;
                    if (k == 0) P.spec_out[M] = Yp;
                }
            }
            if (P.mode & SPEC_MULTIPLY) {
                Yk = cmul(Yk, P.H[k]);
                Yp = cmul(Yp, P.H[k == 0 ? M : M - k]);
            }
            if (P.mode & SPEC_INVERSE) {
                double2 U;
                if (k == 0) {
                    // irfft ignores the imaginary parts of Y[0] and Y[N/2]
                    const double e0 = 0.5 * (Yk.x + Yp.x), o0 = 0.5 * (Yk.x - Yp.x);
                    U = make_double2(e0, o0);
                } else {
                    const double2 Ye = cscale(cadd(Yk, cconj(Yp)), 0.5);
                    const double2 Yo = cmul(twiddle<true>(k, 2LL * M),
                                            cscale(csub(Yk, cconj(Yp)), 0.5));
                    U = cadd(Ye, crot<true>(Yo));     // Ye + i Yo
                }
                other[k2 * Br + br] = U;
            }
        }
        cluster.sync();
        double2* t = rows;
        rows = other;
        other = t;
    }

    if (!(P.mode & SPEC_INVERSE)) return;

    // ---- inverse row transforms (length M2 over k2) -> B[k1][m2]
    double2* rres = batch_fft<true>(rows, other, M2, Br, p.r2, p.n2, tw2);
    double2* rfree = rres == rows ? other : rows;
    cluster.sync();
    // ---- transpose into columns with the conjugate four-step twiddle
    for (int e = tid; e < Bc * M1; e += nth) {
        const int k1 = e % M1, bcol = e / M1;
        const int m2 = c * Bc + bcol;
        const int owner = k1 / Br;
        const double2* remote = cluster.map_shared_rank(rres, owner);
        double2 v = remote[m2 * Br + (k1 - owner * Br)];
        const long long ex = ((long long)k1 * m2) % M;
        if (ex) v = cmul(v, twiddle<true>(ex, M));
        rfree[k1 * Bc + bcol] = v;
    }
    cluster.sync();
    double2* cres = batch_fft<true>(rfree, rres, M1, Bc, p.r1, p.n1, tw1);

    // ---- real output y[2m], y[2m+1] with m = c Bc + b + M2 m1
    double ind = 0.0;
    if (P.ind_coeff) ind = P.ind_coeff[turn];
    const int64_t S = P.n_in;
    for (int e = tid; e < per; e += nth) {
        const int b = e % Bc, m1 = e / Bc;
        const int64_t m = (int64_t)c * Bc + b + (int64_t)M2 * m1;
        const double2 u = cres[m1 * Bc + b];
        const double y2[2] = {u.x, u.y};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int64_t n = 2 * m + h;
            if (n >= P.n_out) continue;
            double v = y2[h] * P.out_scale;
            if (P.ind_coeff) {
                // np.gradient(profile, dbc): central inside, one-sided at ends
                double g;
                if (S < 2) g = 0.0;
                else if (n == 0) g = (P.profile_out[1] - P.profile_out[0]) / P.ind_dbc;
                else if (n == S - 1) g = (P.profile_out[S - 1] - P.profile_out[S - 2]) / P.ind_dbc;
                else g = (P.profile_out[n + 1] - P.profile_out[n - 1]) / (2.0 * P.ind_dbc);
                v = v + ind * g;
            }
            P.out[n] = v;
        }
    }
    if (!P.table && !P.bump_turn) return;
    cluster.sync();  // P.out visible cluster-wide
    if (P.table) {
        const int64_t nt = P.n_out - 1;
        for (int e = tid; e < per; e += nth) {
            const int b = e % Bc, m1 = e / Bc;
            const int64_t m = (int64_t)c * Bc + b + (int64_t)M2 * m1;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int64_t n = 2 * m + h;
                if (n >= nt) continue;
                const double v0 = P.out[n], v1 = P.out[n + 1];
                if (!P.table_f32) {
                    // linear_interp_kick.cpp:44-47 with acc = 0
                    const double slope = P.charge * (v1 - v0) * P.inv_w;
                    const double offset = P.charge * v0 - P.bc[n] * slope;
                    reinterpret_cast<double2*>(P.table)[n] = make_double2(slope, offset);
                } else {
                    reinterpret_cast<float2*>(P.table)[n] =
                        make_float2((float)(P.charge * v0),
                                    (float)(P.charge * (v1 - v0) * P.inv_w));
                }
            }
        }
    }
    if (P.bump_turn && c == 0 && tid == 0) *P.turn = turn + 1;
}

#endif  // BB_SPECTRAL_KERNELS

// Host: choose the factorisation and cluster size for a real length N.
// Returns false when N is odd, too large, or has a prime factor above 5.
bool make_spec_plan(int64_t N, SpecPlan& plan);
// Launch one cluster of spectral_kernel with the plan in P.
int launch_spectral(const SpecParams& P, cudaStream_t stream);
// Set spectral_kernel's launch attributes on the current device (idempotent;
// call before a stream capture that will contain the kernel).
int prepare_spectral();

}  // namespace bb
