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
// from shared tables filled with sincospi() in double precision; the
// four-step and real-to-complex twiddles use a two-level table
// (W^j = A[j / L] * B[j % L]).
//
// Latency is what bounds this kernel, so it is organised around the number
// of cluster barriers: with three buffers per CTA (when they fit) a
// transform never writes the buffer that other CTAs read in the same phase,
// leaving four barriers for the whole rfft -> x Z -> irfft chain; the
// impedance and bin centres are prefetched with cp.async at launch and the
// interpolation table is built from shared memory.
#pragma once

#include <cooperative_groups.h>

#include "common.cuh"
#include "feedback.cuh"

namespace bb {

namespace cg = cooperative_groups;

constexpr int kSpecThreads = 256;  // 8 warps: one per transform in the FFT phases; 255 registers
constexpr int kMaxPasses = 24;
// Largest cluster of the FFT (16: the non-portable maximum); a build may
// define BB_MAX_CLUSTER to compare smaller clusters.
#ifndef BB_MAX_CLUSTER
#define BB_MAX_CLUSTER 16
#endif
constexpr int kMaxCluster = BB_MAX_CLUSTER;
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
    int L;        // split of the two-level twiddle tables (power of two)
    int nbuf;     // 3 (fewer cluster barriers) or 2 (largest lengths)
    int prefetch; // impedance / bin centres staged in shared memory
    int smem;     // dynamic shared memory per CTA, bytes
};

// Bits of SpecParams::mode
enum : int {
    SPEC_FORWARD = 1,     // input is real: pack, forward transform
    SPEC_INVERSE = 2,     // run the inverse transform and write real output
    SPEC_OUT_SPECTRUM = 4,// write the N/2+1 spectrum of the real input
    SPEC_IN_SPECTRUM = 8, // input is an N/2+1 spectrum (irfft only)
    SPEC_MULTIPLY = 16,   // multiply the spectrum by H before inverting
    SPEC_ACCUM = 32,      // acc_g[k] += acc_a[k] * conj(X[k]) over the spectrum
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
    // twiddle tables precomputed for this plan (make_spec_twiddles), or
    // nullptr to compute them in the kernel
    const double2* twg;
    // batch of independent profiles: cluster q (blockIdx.x / C) handles
    // profile q; in_i32 / profile_out / out / bc / table advance by n_in
    // entries per profile, H by M + 1; beam_scale[q] and beam_inv_w[q]
    // replace out_scale and inv_w when given.  No inductive term and no
    // turn reads in batch mode (only the last cluster bumps the counter).
    int batch;
    const double* beam_scale;
    const double* beam_inv_w;
    // SPEC_ACCUM (M + 1 values each): the adjoint of the induced voltage
    // with respect to the impedance needs sum_turns P_t[k] conj(L_t[k]),
    // P_t the profile spectrum and L_t the spectrum of this input
    const double2* acc_a;
    double2* acc_g;
    // launch with programmatic stream serialization (the engine's turn):
    // the kernel triggers its dependents at entry and waits for the grid
    // before it before reading the histogram or the turn counter
    int pdl;
};

// The engine's beam-phase loop run inside the head (single profile only):
// the load phase adds each bin's projections, the CTA that takes the last
// ticket sums the CTAs' warp shares in order and runs the loop.  A separate
// kernel argument, present only in spectral_kernel<true>, so that the
// kernel without the loop is compiled exactly as before.
struct SpecLoop {
    int* ticket;
    FeedbackArgs fb;
};
struct SpecNoLoop {};
template <bool FB> struct SpecLoopArg { using type = SpecNoLoop; };
template <> struct SpecLoopArg<true> { using type = SpecLoop; };

// Device code below is compiled only in spectral.cu (which defines
// BB_SPECTRAL_KERNELS); other files see the types and host entry points.
#ifdef BB_SPECTRAL_KERNELS

// Phase marker for out-of-tree timing builds; expands to nothing here.
#ifndef BB_PHASE
#define BB_PHASE(i)
#endif

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

// ------------------------------------------------------------ radix passes
// The kernel runs each phase a handful of times per launch, so its speed is
// set by instruction fetch (ncu: "no_instruction" was the top stall of a
// version with one inlined pass per radix and direction).  One compact,
// non-inlined pass with a runtime radix and direction serves every
// transform: after its first use it runs from the instruction cache.
//
// multiply by -i (forward, s = -1) or +i (inverse, s = +1)
__device__ __forceinline__ double2 crot_s(double2 a, double s) {
    return make_double2(-s * a.y, s * a.x);
}

// 4-point DFT of (a, b, c, d) in place, sign s of the exponent.
__device__ __forceinline__ void dft4(double2& a, double2& b, double2& c, double2& d, double s) {
    const double2 s02 = cadd(a, c), d02 = csub(a, c);
    const double2 s13 = cadd(b, d), d13 = crot_s(csub(b, d), s);
    a = cadd(s02, s13);
    c = csub(s02, s13);
    b = cadd(d02, d13);
    d = csub(d02, d13);
}

// In-place R-point DFT (R = 2, 3, 4, 5, 8) of v, sign s of the exponent;
// 8 = 2 x 4 (decimation in time).  (A radix-16 butterfly needs enough
// registers to make the kernel spill around the non-inlined pass.)
__device__ __forceinline__ void small_dft(double2* v, int R, double s) {
    if (R == 8) {
        double2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
        double2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
        dft4(e0, e1, e2, e3, s);
        dft4(o0, o1, o2, o3, s);
        const double h = 0.70710678118654752440;
        o1 = cmul(o1, make_double2(h, s * h));
        o2 = crot_s(o2, s);
        o3 = cmul(o3, make_double2(-h, s * h));
        v[0] = cadd(e0, o0);
        v[4] = csub(e0, o0);
        v[1] = cadd(e1, o1);
        v[5] = csub(e1, o1);
        v[2] = cadd(e2, o2);
        v[6] = csub(e2, o2);
        v[3] = cadd(e3, o3);
        v[7] = csub(e3, o3);
        return;
    }
    if (R == 2) {
        const double2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if (R == 4) {
        const double2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
        const double2 s13 = cadd(v[1], v[3]), d13 = crot_s(csub(v[1], v[3]), s);
        v[0] = cadd(s02, s13);
        v[2] = csub(s02, s13);
        v[1] = cadd(d02, d13);
        v[3] = csub(d02, d13);
    } else if (R == 3) {
        const double h = 0.86602540378443864676;  // sin(2 pi / 3)
        const double2 a = v[0], t = cadd(v[1], v[2]), d = csub(v[1], v[2]);
        const double2 m = make_double2(a.x - 0.5 * t.x, a.y - 0.5 * t.y);
        const double2 r = crot_s(cscale(d, h), s);
        v[0] = cadd(a, t);
        v[1] = cadd(m, r);
        v[2] = csub(m, r);
    } else {
        // cos / sin of 2 pi / 5 and 4 pi / 5
        const double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;
        const double s1 = 0.95105651629515357212, s2 = 0.58778525229247312917;
        const double2 a = v[0];
        const double2 t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
        const double2 t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
        const double2 m1 = make_double2(a.x + c1 * t1.x + c2 * t2.x, a.y + c1 * t1.y + c2 * t2.y);
        const double2 m2 = make_double2(a.x + c2 * t1.x + c1 * t2.x, a.y + c2 * t1.y + c1 * t2.y);
        const double2 r1 = crot_s(make_double2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y), s);
        const double2 r2 = crot_s(make_double2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y), s);
        v[0] = cadd(a, cadd(t1, t2));
        v[1] = cadd(m1, r1);
        v[4] = csub(m1, r1);
        v[2] = cadd(m2, r2);
        v[3] = csub(m2, r2);
    }
}

// One Stockham pass of radix R over B interleaved transforms of length L.
// Index arithmetic avoids integer division when the batch count B and the
// stride Ns are powers of two (lgB / lgNs >= 0): every power-of-two length,
// i.e. every next_regular result of the usual 2^k slice counts.
__device__ __noinline__ void stockham_pass(const double2* __restrict__ src,
                                           double2* __restrict__ dst, int L, int B,
                                           int Ns, int R, const double2* __restrict__ tw,
                                           double s, int lgB, int lgNs, int LR, int step) {
    const int total = B * LR;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int b = lgB >= 0 ? (idx & (B - 1)) : idx % B;
        const int j = lgB >= 0 ? (idx >> lgB) : idx / B;
        const int k = lgNs >= 0 ? (j & (Ns - 1)) : j % Ns;
        const int jq = lgNs >= 0 ? (j >> lgNs) : j / Ns;
        double2 v[8];
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            if (t < R) {
                double2 x = src[(j + t * LR) * B + b];
                if (t > 0 && k > 0) {
                    double2 w = tw[t * k * step];
                    w.y = -s * w.y;  // table holds exp(-2 pi i q / L)
                    x = cmul(x, w);
                }
                v[t] = x;
            }
        }
        small_dft(v, R, s);
        const int d = jq * Ns * R + k;
#pragma unroll
        for (int t = 0; t < 8; ++t)
            if (t < R) dst[(d + t * Ns) * B + b] = v[t];
    }
}

// B transforms of length L = 32 P (P = 1, 2, 4, 8) held interleaved in a
// (element (b, i) at a[i * B + b]), transformed in place with one warp per
// transform: lane l holds elements l + 32 q (q < P) in registers; radix-2
// decimation in frequency, the butterflies of span >= 32 inside a lane, the
// spans 16 .. 1 across lanes with shuffles (no block barrier inside a
// transform), the results written back in natural order (the output of
// decimation in frequency sits at the bit-reversed index).  tw[q] =
// exp(-2 pi i q / L); the inverse uses the conjugates.  The Stockham passes
// keep only 2-4 warps of a block busy, each on a long dependent chain, and
// need a block barrier per pass; here every transform is one warp's
// register-resident work.  Ends with __syncthreads().
template <int P>
__device__ __forceinline__ void warp_fft(double2* a, int B, const double2* __restrict__ tw,
                                      bool inverse, int lgL) {
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int L = 32 * P;
    const double sg = inverse ? -1.0 : 1.0;  // sign of the twiddles' imaginary parts
    for (int b = threadIdx.x >> 5; b < B; b += nw) {
        double2 v[P];
#pragma unroll
        for (int q = 0; q < P; ++q) v[q] = a[(lane + 32 * q) * B + b];
        // spans h = 32 hq >= 32: both elements in this lane
#pragma unroll
        for (int hq = P / 2; hq >= 1; hq >>= 1) {
#pragma unroll
            for (int q = 0; q < P; ++q) {
                if (q & hq) continue;
                const int i = lane + 32 * q;  // the pair's lower index
                const int e = (i & (64 * hq - 1)) * (L / (64 * hq));
                double2 w = tw[e];
                w.y *= sg;
                const double2 x = v[q], y = v[q + hq];
                v[q] = cadd(x, y);
                v[q + hq] = cmul(csub(x, y), w);
            }
        }
        // spans h = 16 .. 1: the partner is lane l ^ h
#pragma unroll
        for (int h = 16; h >= 1; h >>= 1) {
            const bool upper = (lane & h) != 0;
            double2 w = upper ? tw[(lane & (h - 1)) * (L / (2 * h))] : make_double2(1.0, 0.0);
            w.y *= sg;
#pragma unroll
            for (int q = 0; q < P; ++q) {
                double2 p;
                p.x = __shfl_xor_sync(0xffffffffu, v[q].x, h);
                p.y = __shfl_xor_sync(0xffffffffu, v[q].y, h);
                v[q] = upper ? cmul(csub(p, v[q]), w) : cadd(v[q], p);
            }
        }
#pragma unroll
        for (int q = 0; q < P; ++q) {
            const int k = (int)(__brev((unsigned)(lane + 32 * q)) >> (32 - lgL));
            a[k * B + b] = v[q];
        }
    }
    __syncthreads();
}

// B transforms of length G = 2, 4, 8 or 16 (interleaved as in warp_fft):
// a group of G lanes per transform, one element per lane, 32 / G
// transforms per warp; the butterflies of every span by shuffles inside the
// group, radix-2 decimation in frequency, results to the bit-reversed
// index.  Replaces the Stockham passes (a block barrier each) for the short
// factors of small plans (512- and 1024-point transforms).  Ends with
// __syncthreads().
template <int G>
__device__ __forceinline__ void subwarp_fft(double2* a, int B, const double2* __restrict__ tw,
                                            bool inverse, int lgG) {
    const int lane = threadIdx.x & 31, gl = lane & (G - 1), grp = lane / G;
    const int tpw = 32 / G, nw = blockDim.x >> 5;
    const double sg = inverse ? -1.0 : 1.0;
    // b0 is the same for the whole warp, so every lane reaches the shuffles
    for (int b0 = (threadIdx.x >> 5) * tpw; b0 < B; b0 += nw * tpw) {
        const int b = b0 + grp;
        const bool act = b < B;
        double2 v = act ? a[gl * B + b] : make_double2(0.0, 0.0);
#pragma unroll
        for (int h = G / 2; h >= 1; h >>= 1) {
            const bool upper = (gl & h) != 0;
            double2 w = upper ? tw[(gl & (h - 1)) * (G / (2 * h))] : make_double2(1.0, 0.0);
            w.y *= sg;
            double2 q;
            q.x = __shfl_xor_sync(0xffffffffu, v.x, h);
            q.y = __shfl_xor_sync(0xffffffffu, v.y, h);
            v = upper ? cmul(csub(q, v), w) : cadd(v, q);
        }
        if (act) a[(int)(__brev((unsigned)gl) >> (32 - lgG)) * B + b] = v;
    }
    __syncthreads();
}

// The register transforms of lengths 32 .. 256 in place.  Not inlined: the
// head calls the transform batch six times, and six inlined copies of these
// made the kernel's code about 700 KB, whose instruction fetches were the
// head's top stall.
__device__ __noinline__ void warp_fft_any(double2* a, int L, int B, const double2* tw,
                                          bool inverse) {
    switch (L) {
        case 2: subwarp_fft<2>(a, B, tw, inverse, 1); return;
        case 4: subwarp_fft<4>(a, B, tw, inverse, 2); return;
        case 8: subwarp_fft<8>(a, B, tw, inverse, 3); return;
        case 16: subwarp_fft<16>(a, B, tw, inverse, 4); return;
        case 32: warp_fft<1>(a, B, tw, inverse, 5); return;
        case 64: warp_fft<2>(a, B, tw, inverse, 6); return;
        case 128: warp_fft<4>(a, B, tw, inverse, 7); return;
        default: warp_fft<8>(a, B, tw, inverse, 8); return;
    }
}

// B transforms of length L, interleaved, starting in a[]; returns the buffer
// (a or b) that holds the result.  Ends with __syncthreads().
__device__ double2* batch_fft(double2* a, double2* b, int L, int B, const int* radices,
                              int npass, const double2* tw, bool inverse) {
    if (L >= 2 && L <= 256 && (L & (L - 1)) == 0) {
        warp_fft_any(a, L, B, tw, inverse);
        return a;
    }
    const double s = inverse ? 1.0 : -1.0;
    const int lgB = (B & (B - 1)) == 0 ? __ffs(B) - 1 : -1;
    int Ns = 1;
    for (int p = 0; p < npass; ++p) {
        const int R = radices[p];
        const int lgNs = (Ns & (Ns - 1)) == 0 ? __ffs(Ns) - 1 : -1;
        stockham_pass(a, b, L, B, Ns, R, tw, s, lgB, lgNs, L / R, L / (Ns * R));
        __syncthreads();
        double2* t = a;
        a = b;
        b = t;
        Ns *= R;
    }
    return a;
}

// The six twiddle tables of a plan (contiguous in the shared layout, and in
// the same order in a precomputed global copy): tw1[q] = W_M1^q,
// tw2[q] = W_M2^q, tam[a] = W_M^(aL), tbm[b] = W_M^b, tan[a] = W_N^(aL),
// tbn[b] = W_N^b, with W_X = exp(-2 pi i / X) from sincospi.
__device__ inline void fill_twiddles(const SpecPlan& p, double2* tw1, double2* tw2,
                                     double2* tam, double2* tbm, double2* tan_,
                                     double2* tbn, int tid, int nth) {
    const int M = p.M, L = p.L, nA = (M + L - 1) / L;
    for (int q = tid; q < p.M1; q += nth) tw1[q] = twiddle<false>(q, p.M1);
    for (int q = tid; q < p.M2; q += nth) tw2[q] = twiddle<false>(q, p.M2);
    for (int q = tid; q < nA; q += nth) {
        tam[q] = twiddle<false>((long long)q * L, M);
        tan_[q] = twiddle<false>((long long)q * L, 2LL * M);
    }
    for (int q = tid; q < L; q += nth) {
        tbm[q] = twiddle<false>(q, M);
        tbn[q] = twiddle<false>(q, 2LL * M);
    }
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}

// Shared-memory carve-up of one CTA (offsets in bytes), shared with the host.
struct SpecLayout {
    int bufs, tw1, tw2, tam, tbm, tan_, tbn, hk, hp, bcs, vloc, nbr, total;
};
__host__ __device__ inline SpecLayout spec_layout(const SpecPlan& p) {
    SpecLayout s;
    const int per = p.M / p.C, nA = (p.M + p.L - 1) / p.L;
    int o = 0;
    s.bufs = o; o += 16 * p.nbuf * per;
    s.tw1 = o;  o += 16 * p.M1;
    s.tw2 = o;  o += 16 * p.M2;
    s.tam = o;  o += 16 * nA;
    s.tbm = o;  o += 16 * p.L;
    s.tan_ = o; o += 16 * nA;
    s.tbn = o;  o += 16 * p.L;
    s.hk = o;   o += p.prefetch ? 16 * per : 0;
    s.hp = o;   o += p.prefetch ? 16 * per : 0;
    s.bcs = o;  o += p.prefetch ? 16 * per : 0;  // two doubles per element
    s.vloc = o; o += 8 * per;
    s.nbr = o;  o += 8 * p.M1;
    s.total = o;
    return s;
}

// ------------------------------------------------------------ the kernel
// One cluster of p.C CTAs.  Column phase: CTA c owns n2 in [c Bc, (c+1) Bc),
// element (n1, n2) at n1 * Bc + n2 - c Bc.  Row phase: CTA c owns k1 in
// [c Br, (c+1) Br), element (k1, k2) at k2 * Br + k1 - c Br.
template <bool FB>
__global__ void __launch_bounds__(kSpecThreads, 1)
spectral_kernel(const SpecParams P, const typename SpecLoopArg<FB>::type LP) {
    cg::cluster_group cluster = cg::this_cluster();
    pdl_launch_dependents();  // the particle pass may launch and set up now
    const SpecPlan& p = P.p;
    const int c = (int)cluster.block_rank();
    const int tid = threadIdx.x, nth = blockDim.x;
    extern __shared__ __align__(16) unsigned char sraw[];
    const SpecLayout lay = spec_layout(p);
    const int per = p.M / p.C;
    const int M = p.M, M1 = p.M1, M2 = p.M2, Bc = p.Bc, Br = p.Br, L = p.L;
    // this cluster's profile (batch mode) and its arrays
    const int beam = P.batch ? (int)(blockIdx.x / p.C) : 0;
    const int64_t boff = (int64_t)beam * P.n_in;
    int* const g_in_i32 = P.in_i32 ? P.in_i32 + boff : nullptr;
    const double* const g_in_f64 = P.in_f64 ? P.in_f64 + boff : nullptr;
    double* const g_profile = P.profile_out ? P.profile_out + boff : nullptr;
    double* const g_out = P.out ? P.out + boff : nullptr;
    const double* const g_bc = P.bc ? P.bc + boff : nullptr;
    void* const g_table =
        P.table ? static_cast<char*>(P.table) + boff * (P.table_f32 ? 8 : 16) : nullptr;
    const double2* const g_H = P.H ? P.H + (int64_t)beam * (M + 1) : nullptr;
    const double out_scale = P.beam_scale ? P.beam_scale[beam] : P.out_scale;
    const double inv_w = P.beam_inv_w ? P.beam_inv_w[beam] : P.inv_w;
    double2* buf[3] = {reinterpret_cast<double2*>(sraw + lay.bufs),
                       reinterpret_cast<double2*>(sraw + lay.bufs) + per,
                       reinterpret_cast<double2*>(sraw + lay.bufs) + 2 * per};
    double2* tw1 = reinterpret_cast<double2*>(sraw + lay.tw1);
    double2* tw2 = reinterpret_cast<double2*>(sraw + lay.tw2);
    double2* tam = reinterpret_cast<double2*>(sraw + lay.tam);
    double2* tbm = reinterpret_cast<double2*>(sraw + lay.tbm);
    double2* tan_ = reinterpret_cast<double2*>(sraw + lay.tan_);
    double2* tbn = reinterpret_cast<double2*>(sraw + lay.tbn);
    double2* hk = reinterpret_cast<double2*>(sraw + lay.hk);
    double2* hp = reinterpret_cast<double2*>(sraw + lay.hp);
    double* bcs = reinterpret_cast<double*>(sraw + lay.bcs);
    double* vloc = reinterpret_cast<double*>(sraw + lay.vloc);
    double* nbr = reinterpret_cast<double*>(sraw + lay.nbr);
    const bool three = p.nbuf == 3;
    const bool inverse = (P.mode & SPEC_INVERSE) != 0;
    // Index arithmetic without runtime integer division where the factors
    // are powers of two (every plan of a power-of-two n_fft): quotient and
    // remainder by shift and mask.  L always is one.
    const bool pw = (M1 & (M1 - 1)) == 0 && (M2 & (M2 - 1)) == 0 && (Bc & (Bc - 1)) == 0 &&
                    (Br & (Br - 1)) == 0;
    const int lgM1 = 31 - __clz(M1), lgM2 = 31 - __clz(M2);
    const int lgBc = 31 - __clz(Bc), lgBr = 31 - __clz(Br), lgL = 31 - __clz(L);
    auto qr = [&](int x, int d, int lg, int& q, int& r) {
        if (pw) {
            q = x >> lg;
            r = x & (d - 1);
        } else {
            q = x / d;
            r = x - q * d;
        }
    };

    BB_PHASE(0);
    // ---- twiddle tables precomputed by the engine: copied asynchronously
    // (one contiguous block tw1 .. tbn of the layout), first group
    if (P.twg) {
        double2* dst = reinterpret_cast<double2*>(sraw + lay.tw1);
        const int cnt = (lay.hk - lay.tw1) / 16;
        for (int q = tid; q < cnt; q += nth) cp_async16(&dst[q], &P.twg[q]);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    // ---- prefetch what later phases read from global memory
    if (p.prefetch) {
        if (P.mode & SPEC_MULTIPLY) {
            for (int e = tid; e < per; e += nth) {
                int q, r;
                qr(e, Br, lgBr, q, r);
                const int k = c * Br + r + M1 * q;
                cp_async16(&hk[e], &g_H[k]);
                cp_async16(&hp[e], &g_H[k == 0 ? M : M - k]);
            }
        }
        if (inverse && g_table) {
            for (int e = tid; e < per; e += nth) {
                int q, r;
                qr(e, Bc, lgBc, q, r);
                const int64_t m = (int64_t)c * Bc + r + (int64_t)M2 * q;
                if (2 * m < P.n_out - 1) cp_async8(&bcs[2 * e], &g_bc[2 * m]);
                if (2 * m + 1 < P.n_out - 1) cp_async8(&bcs[2 * e + 1], &g_bc[2 * m + 1]);
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    pdl_wait();  // the previous grid's histogram, counter and programme
    const long long turn = P.turn ? *P.turn : 0;
    double ind = 0.0;
    if (P.ind_coeff) ind = P.ind_coeff[turn];
    bool fb_on = false;
    double fb_s = 0, fb_c = 0;
    FbBins fbb = {};
    if constexpr (FB) {
        fb_on = turn >= LP.fb.delay;
        if (fb_on) fbb = fb_bins(LP.fb, turn);
    }

    BB_PHASE(1);
    // ---- twiddle tables (computed here unless they were copied)
    if (!P.twg) fill_twiddles(p, tw1, tw2, tam, tbm, tan_, tbn, tid, nth);
    // the copied tables must have landed before the first transform;
    // the prefetch group (if any) may still be in flight
    auto wait_twiddles = [&]() {
        if (P.twg) {
            if (p.prefetch) asm volatile("cp.async.wait_group 1;" ::: "memory");
            else asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
    };
    // W_M^j and W_N^j (N = 2M) for 0 <= j < M from the two-level tables
    // (0 <= j < M: int arithmetic, L a power of two)
    auto twm = [&](int j) { return cmul(tam[j >> lgL], tbm[j & (L - 1)]); };
    auto twn = [&](int j) { return cmul(tan_[j >> lgL], tbn[j & (L - 1)]); };

    double2* rows = nullptr;   // row-phase buffer holding Z
    double2* spare = nullptr;  // buffers that no other CTA reads right now
    double2* spare2 = nullptr;

    if (P.mode & SPEC_FORWARD) {
        BB_PHASE(2);
        // ---- load: z[m] = x[2m] + i x[2m+1], m = c Bc + b + M2 n1
        const int64_t nlim = P.n_in < (int64_t)p.N ? P.n_in : (int64_t)p.N;
        for (int e = tid; e < per; e += nth) {
            int n1, b;
            qr(e, Bc, lgBc, n1, b);
            const int64_t m = (int64_t)c * Bc + b + (int64_t)M2 * n1;
            double x0 = 0.0, x1 = 0.0;
            const int64_t i0 = 2 * m, i1 = 2 * m + 1;
            if (g_in_i32) {
                if (i0 < nlim) { x0 = (double)g_in_i32[i0]; g_in_i32[i0] = 0; }
                if (i1 < nlim) { x1 = (double)g_in_i32[i1]; g_in_i32[i1] = 0; }
                if (g_profile) {
                    if (i0 < P.n_in) g_profile[i0] = x0;
                    if (i1 < P.n_in) g_profile[i1] = x1;
                }
                if (fb_on) {
                    if (i0 < nlim) fb_add(fbb, (int)i0, x0, fb_s, fb_c);
                    if (i1 < nlim) fb_add(fbb, (int)i1, x1, fb_s, fb_c);
                }
            } else {
                if (i0 < nlim) x0 = g_in_f64[i0];
                if (i1 < nlim) x1 = g_in_f64[i1];
            }
            buf[0][n1 * Bc + b] = make_double2(x0, x1);
        }
        // histogram bins beyond the transform length (profile longer than
        // n_fft): converted and cleared but not transformed
        if (g_in_i32 && c == 0) {
            for (int64_t i = (int64_t)p.N + tid; i < P.n_in; i += nth) {
                const double x = (double)g_in_i32[i];
                g_in_i32[i] = 0;
                if (g_profile) g_profile[i] = x;
                if (fb_on) fb_add(fbb, (int)i, x, fb_s, fb_c);
            }
        }
        wait_twiddles();
        __syncthreads();
        BB_PHASE(3);
        // ---- column transforms (length M1 over n1, Bc of them)
        double2* r1 = batch_fft(buf[0], buf[1], M1, Bc, p.r1, p.n1, tw1, false);
        double2* f1 = r1 == buf[0] ? buf[1] : buf[0];
        BB_PHASE(4);
        cluster.sync();  // (A) every CTA's columns done
        BB_PHASE(5);
        // ---- transpose into rows with the four-step twiddle W_M^(n2 k1),
        // written to a buffer nobody reads remotely
        for (int e = tid; e < Br * M2; e += nth) {
            int br, n2;
            qr(e, M2, lgM2, br, n2);
            const int k1 = c * Br + br;
            int owner, nl;
            qr(n2, Bc, lgBc, owner, nl);
            const double2* remote = cluster.map_shared_rank(r1, owner);
            double2 v = remote[k1 * Bc + nl];
            const int ex = n2 * k1;  // < M1 M2 = M
            if (ex) v = cmul(v, twm(ex));
            f1[n2 * Br + br] = v;
        }
        // with two buffers the row transform would overwrite r1 while other
        // CTAs may still read it
        if (three) {
            __syncthreads();
            BB_PHASE(6);
            rows = batch_fft(f1, buf[2], M2, Br, p.r2, p.n2, tw2, false);
            spare = rows == f1 ? buf[2] : f1;
            spare2 = r1;
            BB_PHASE(7);
        } else {
            cluster.sync();
            rows = batch_fft(f1, r1, M2, Br, p.r2, p.n2, tw2, false);
            spare = rows == f1 ? r1 : f1;
        }
        cluster.sync();  // (C) Z complete everywhere
        BB_PHASE(8);
    } else {
        wait_twiddles();
        __syncthreads();  // twiddle tables
        spare = buf[0];
        spare2 = three ? buf[2] : nullptr;
    }

    if (p.prefetch) asm volatile("cp.async.wait_group 0;" ::: "memory");
    BB_PHASE(9);

    double2* ubuf = nullptr;
    if (P.mode & (SPEC_OUT_SPECTRUM | SPEC_MULTIPLY | SPEC_IN_SPECTRUM)) {
        // ---- spectral step on own k = k1 + M1 k2 with partner M - k
        ubuf = spare;
        for (int e = tid; e < per; e += nth) {
            int k2, br;
            qr(e, Br, lgBr, k2, br);
            const int k1 = c * Br + br;
            const int k = k1 + M1 * k2;
            const int pk = k == 0 ? 0 : M - k;
            double2 Yk, Yp;  // Y[k], Y[M-k] (Y[M] when k == 0)
            if (P.mode & SPEC_IN_SPECTRUM) {
                const int64_t kk = k, kp = (k == 0) ? M : (M - k);
                Yk = kk < P.n_spec_in ? P.spec_in[kk] : make_double2(0, 0);
                Yp = kp < P.n_spec_in ? P.spec_in[kp] : make_double2(0, 0);
            } else {
                int p2, p1, owner, pl;
                qr(pk, M1, lgM1, p2, p1);
                qr(p1, Br, lgBr, owner, pl);
                const double2* remote = cluster.map_shared_rank(rows, owner);
                const double2 Zk = rows[k2 * Br + br];
                const double2 Zp = remote[p2 * Br + pl];
                if (k == 0) {
                    Yk = make_double2(Zk.x + Zk.y, 0.0);  // X[0]
                    Yp = make_double2(Zk.x - Zk.y, 0.0);  // X[M]
                } else {
                    const double2 E = cscale(cadd(Zk, cconj(Zp)), 0.5);
                    const double2 O = crot<false>(cscale(csub(Zk, cconj(Zp)), 0.5));
                    const double2 wO = cmul(twn(k), O);  // e^{-2 pi i k/N} O
                    Yk = cadd(E, wO);                    // X[k]
                    Yp = cconj(csub(E, wO));             // X[M-k]
                }
                if (P.mode & SPEC_OUT_SPECTRUM) {
                    // every k < M is owned once; X[M] comes from k == 0
                    P.spec_out[k] = Yk;
                    if (k == 0) P.spec_out[M] = Yp;
                }
                if (P.mode & SPEC_ACCUM) {
                    P.acc_g[k] = cadd(P.acc_g[k], cmul(P.acc_a[k], cconj(Yk)));
                    if (k == 0) P.acc_g[M] = cadd(P.acc_g[M], cmul(P.acc_a[M], cconj(Yp)));
                }
            }
            if (P.mode & SPEC_MULTIPLY) {
                const double2 Hk = p.prefetch ? hk[e] : g_H[k];
                const double2 Hp = p.prefetch ? hp[e] : g_H[k == 0 ? M : M - k];
                Yk = cmul(Yk, Hk);
                Yp = cmul(Yp, Hp);
            }
            if (inverse) {
                double2 U;
                if (k == 0) {
                    // irfft ignores the imaginary parts of Y[0] and Y[N/2]
                    const double e0 = 0.5 * (Yk.x + Yp.x), o0 = 0.5 * (Yk.x - Yp.x);
                    U = make_double2(e0, o0);
                } else {
                    const double2 Ye = cscale(cadd(Yk, cconj(Yp)), 0.5);
                    const double2 Yo = cmul(cconj(twn(k)), cscale(csub(Yk, cconj(Yp)), 0.5));
                    U = cadd(Ye, crot<true>(Yo));     // Ye + i Yo
                }
                ubuf[k2 * Br + br] = U;
            }
        }
    }
    BB_PHASE(10);
    if (!inverse) {
        cluster.sync();  // partners' reads of `rows` done before this CTA exits
        return;
    }

    // ---- inverse row transforms (length M2 over k2) -> B[k1][m2], never
    // touching `rows`, which partners may still read (three buffers), or
    // after a barrier (two)
    double2* rres;
    double2* rfree;
    if (three || !rows) {
        double2* other = three ? spare2 : buf[1];
        __syncthreads();
        rres = batch_fft(ubuf, other, M2, Br, p.r2, p.n2, tw2, true);
        rfree = rres == ubuf ? other : ubuf;
        BB_PHASE(11);
    } else {
        cluster.sync();
        rres = batch_fft(ubuf, rows, M2, Br, p.r2, p.n2, tw2, true);
        rfree = rres == ubuf ? rows : ubuf;
    }
    cluster.sync();  // (E) every CTA's rows done
    BB_PHASE(12);
    // ---- transpose into columns with the conjugate four-step twiddle
    double2* cdst = (three && rows) ? rows : rfree;  // rows is free after (E)
    for (int e = tid; e < Bc * M1; e += nth) {
        int bcol, k1;
        qr(e, M1, lgM1, bcol, k1);
        const int m2 = c * Bc + bcol;
        int owner, kl;
        qr(k1, Br, lgBr, owner, kl);
        const double2* remote = cluster.map_shared_rank(rres, owner);
        double2 v = remote[m2 * Br + kl];
        const int ex = k1 * m2;  // < M
        if (ex) v = cmul(v, cconj(twm(ex)));
        cdst[k1 * Bc + bcol] = v;
    }
    double2* cres;
    if (three && rows) {
        __syncthreads();
        cres = batch_fft(cdst, rfree, M1, Bc, p.r1, p.n1, tw1, true);
    } else {
        cluster.sync();
        cres = batch_fft(cdst, rres, M1, Bc, p.r1, p.n1, tw1, true);
    }

    BB_PHASE(13);
    // ---- real output y[2m], y[2m+1] with m = c Bc + b + M2 m1
    const int64_t S = P.n_in;
    auto value = [&](int64_t n, double y) {
        double v = y * out_scale;
        if (P.ind_coeff) {
            // np.gradient(profile, dbc): central inside, one-sided at ends
            double g;
            if (S < 2) g = 0.0;
            else if (n == 0) g = (g_profile[1] - g_profile[0]) / P.ind_dbc;
            else if (n == S - 1) g = (g_profile[S - 1] - g_profile[S - 2]) / P.ind_dbc;
            else g = (g_profile[n + 1] - g_profile[n - 1]) / (2.0 * P.ind_dbc);
            v = v + ind * g;
        }
        return v;
    };
    for (int e = tid; e < per; e += nth) {
        int m1, b;
        qr(e, Bc, lgBc, m1, b);
        const int64_t m = (int64_t)c * Bc + b + (int64_t)M2 * m1;
        const double2 u = cres[m1 * Bc + b];
        const double v0 = value(2 * m, u.x), v1 = value(2 * m + 1, u.y);
        if (2 * m < P.n_out) g_out[2 * m] = v0;
        if (2 * m + 1 < P.n_out) g_out[2 * m + 1] = v1;
        if (g_table) {
            vloc[e] = v0;
            // v0 is V[2(m-1)+2] for the element before m: hand it to the
            // CTA that owns that element (first column of a CTA only)
            if (b == 0 && m > 0) {
                if (c > 0) cluster.map_shared_rank(nbr, c - 1)[m1] = v0;
                else cluster.map_shared_rank(nbr, p.C - 1)[m1 - 1] = v0;
            }
        }
    }
    // (G) the neighbour values have landed, and every CTA has finished
    // reading the others' `rres` -- no CTA may exit before that
    cluster.sync();
    BB_PHASE(14);
    if (!g_table && !P.bump_turn) return;
    if (g_table) {
        const int64_t nt = P.n_out - 1;
        for (int e = tid; e < per; e += nth) {
            int m1, b;
        qr(e, Bc, lgBc, m1, b);
            const int64_t m = (int64_t)c * Bc + b + (int64_t)M2 * m1;
            const double2 u = cres[m1 * Bc + b];
            const double v0 = vloc[e];
            const double v1 = value(2 * m + 1, u.y);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int64_t n = 2 * m + h;
                if (n >= nt) continue;
                const double a0 = h == 0 ? v0 : v1;
                const double a1 = h == 0 ? v1 : (b + 1 < Bc ? vloc[e + 1] : nbr[m1]);
                const double bcn = p.prefetch ? bcs[2 * e + h] : g_bc[n];
                if (!P.table_f32) {
                    // linear_interp_kick.cpp:44-47 with acc = 0
                    reinterpret_cast<double2*>(g_table)[n] =
                        lik_entry0(a0, a1, bcn, P.charge, inv_w);
                } else {
                    reinterpret_cast<float2*>(g_table)[n] =
                        make_float2((float)(P.charge * a0),
                                    (float)(P.charge * (a1 - a0) * inv_w));
                }
            }
        }
    }
    if constexpr (FB) {
        // the CTAs' warp shares, then the last CTA runs this turn's loop
        for (int d = 16; d > 0; d >>= 1) {
            fb_s += __shfl_down_sync(0xffffffffu, fb_s, d);
            fb_c += __shfl_down_sync(0xffffffffu, fb_c, d);
        }
        const int lane = tid & 31, wpb = nth >> 5;
        if (lane == 0) {
            LP.fb.phase_partials[2 * (c * wpb + (tid >> 5))] = fb_s;
            LP.fb.phase_partials[2 * (c * wpb + (tid >> 5)) + 1] = fb_c;
            __threadfence();
        }
        __syncthreads();
        int last = 0;
        if (tid == 0) last = atomicAdd(LP.ticket, 1) == p.C - 1;
        last = __syncthreads_or(last);
        if (last && tid < 32) {
            __threadfence();
            double s = 0, cc = 0, dsum = 0;
            for (int q = lane; q < p.C * wpb; q += 32) {
                s += LP.fb.phase_partials[2 * q];
                cc += LP.fb.phase_partials[2 * q + 1];
            }
            if (LP.fb.machine == BLOND_FB_SPS_RL && fb_on)
                for (int q = lane; q < kFbPartials; q += 32) dsum += LP.fb.partials[q];
            for (int d = 16; d > 0; d >>= 1) {
                s += __shfl_down_sync(0xffffffffu, s, d);
                cc += __shfl_down_sync(0xffffffffu, cc, d);
                dsum += __shfl_down_sync(0xffffffffu, dsum, d);
            }
            if (lane == 0) {
                *LP.ticket = 0;
                fb_turn_end(LP.fb, turn, s, cc, dsum);
            }
        }
    }
    if (P.bump_turn && beam == 0 && c == 0 && tid == 0) *P.turn = turn + 1;
    BB_PHASE(15);
}

#endif  // BB_SPECTRAL_KERNELS

// Host: choose the factorisation and cluster size for a real length N.
// Returns false when N is odd, too large, or has a prime factor above 5.
bool make_spec_plan(int64_t N, SpecPlan& plan, int max_cluster = kMaxCluster);
// Launch one cluster of spectral_kernel with the plan in P.
int launch_spectral(const SpecParams& P, cudaStream_t stream);
// The same with the engine's beam-phase loop inside (single profile).
int launch_spectral_loop(const SpecParams& P, const SpecLoop& L, cudaStream_t stream);
// Set spectral_kernel's launch attributes on the current device (idempotent;
// call before a stream capture that will contain the kernel).
int prepare_spectral();
// Allocate (cudaMalloc) and fill the twiddle tables of a plan for
// SpecParams::twg; the caller frees *out with cudaFree.  Synchronous.
int make_spec_twiddles(const SpecPlan& plan, double2** out);

}  // namespace bb
