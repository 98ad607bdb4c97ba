// Fused per-turn tracking engine.
//
// One turn of the reference main loop [TotalInducedVoltage, RingAndRFTracker,
// Profile] (EX_05_Wake_impedance.py:318-339) touches every particle four
// times in the reference (lik, kick, drift, histogram: 80 B per particle in
// FP64).  Here it is two launches:
//
//   head      one cluster (spectral_kernel) or one CTA: profile <- histogram
//             (and clears it), induced voltage + interpolation table for this
//             turn, turn counter += 1;
//   particles one pass over SoA dt/dE: interpolated induced kick, RF kick of
//             turn t, drift with turn t+1 parameters, deposit into a
//             shared-memory histogram flushed with integer atomics --
//             32 B per particle in FP64 (24 B in F32P64).
//
// The turn index lives in device memory, so a CUDA graph of K turns is
// captured once and replayed.
#include "spectral.cuh"
#include "feedback.cuh"

#include <algorithm>
#include <cstddef>
#include <mutex>
#include <set>
#include <utility>
#include <vector>

namespace bb {

constexpr int kMaxRfEngine = 16;

struct DriftTurn {
    double Tr;      // t_rev * length_ratio
    double simple;  // Tr * eta_0 / (beta^2 E)
    double e0, e1, e2;
    double ib2, ie2, energy;
    double a0, a1, a2;
    double pad;
};

struct ParticleArgs {
    void* dt;
    void* dE;
    int64_t n;
    int n_rf;
    double charge;
    const double* V;    // [(turns+1) * n_rf]
    const double* om;
    const double* ph;
    const double* acc;  // [turns]
    const DriftTurn* drift;  // [turns+1]
    int order;          // legacy alpha order
    int64_t n_turns;
    const long long* turn;
    // slicing
    int S;
    double cut_left, inv_w;
    int* hist;
    // interpolation table (induced voltage)
    const void* table;
    double bc0, lik_inv_w, bw;
    int global_hist;  // 1: deposit into `hist` directly (no shared copy)
    int tma_stages;   // chunks in flight per block of the staged pass
};

enum { PREC_F64 = 0, PREC_F32P64 = 1 };

template <int PREC>
struct Coord;
template <> struct Coord<PREC_F64> { using E = double; };
template <> struct Coord<PREC_F32P64> { using E = float; };

struct TurnConsts {
    double V[kMaxRfEngine], om[kMaxRfEngine], ph[kMaxRfEngine];
    float Vf[kMaxRfEngine];
    double acc;
    DriftTurn d;
};

// 2 pi split for the FP64 range reduction of the RF phase.
__device__ __forceinline__ double reduce_2pi(double x) {
    const double inv2pi = 0.15915494309189533577;
    const double twopi = 6.28318530717958647692;
    return fma(-rint(x * inv2pi), twopi, x);
}

template <int PREC, int SOLVER, bool LIK, bool KICK, bool HIST, bool WARP_AGG>
__device__ __forceinline__ void track_one(double& t,
                                          typename Coord<PREC>::E& e,
                                          const TurnConsts& c,
                                          const ParticleArgs& a, int* sh, int order) {
    using E = typename Coord<PREC>::E;
    if (KICK) {
        if (LIK) {
            const double f = floor((t - a.bc0) * a.lik_inv_w);
            if (f >= 0.0 && f < (double)(a.S - 1)) {
                const int k = (int)f;
                if (PREC == PREC_F64) {
                    const double2 tb = __ldg(reinterpret_cast<const double2*>(a.table) + k);
                    e += t * tb.x + tb.y;
                } else {
                    const float2 tb = __ldg(reinterpret_cast<const float2*>(a.table) + k);
                    const float x = (float)(t - (a.bc0 + (double)k * a.bw));
                    e += __fmaf_rn(tb.y, x, tb.x);
                }
            }
        }
        if (PREC == PREC_F64) {
            double s = 0.0;
            for (int j = 0; j < a.n_rf; ++j) s += c.V[j] * sin(c.om[j] * t + c.ph[j]);
            e += a.charge * s + c.acc;
        } else {
            float s = 0.0f;
            for (int j = 0; j < a.n_rf; ++j)
                s += c.Vf[j] * sinf((float)reduce_2pi(fma(c.om[j], t, c.ph[j])));
            e += (float)a.charge * s + (float)c.acc;
        }
        // dt accumulates in float64 in both precision modes
        if (SOLVER == BLOND_SOLVER_SIMPLE)
            t = drift_simple<double>(t, (double)e, c.d.simple);
        else if (SOLVER == BLOND_SOLVER_LEGACY)
            t = drift_legacy<double>(t, (double)e, c.d.Tr, c.d.e0, c.d.e1, c.d.e2, order);
        else
            t = drift_exact<double>(t, (double)e, c.d.Tr, c.d.ib2, c.d.ie2, c.d.a0, c.d.a1,
                                    c.d.a2, c.d.energy);
    }
    (void)sh;
}

// Two particles at once, with the interpolation-table gathers (L2-resident,
// the longest-latency loads of the pass) issued before the RF sines so their
// latency overlaps the sine arithmetic.  Same operations, in the same order
// per particle, as two calls of track_one.
template <int PREC, int SOLVER, bool LIK>
__device__ __forceinline__ void track_pair(double& t0, double& t1,
                                           typename Coord<PREC>::E& e0,
                                           typename Coord<PREC>::E& e1,
                                           const TurnConsts& c, const ParticleArgs& a,
                                           int order) {
    using E = typename Coord<PREC>::E;
    using TB = typename Vec2<E>::type;
    bool in0 = false, in1 = false;
    TB tb0, tb1;
    float x0f = 0.0f, x1f = 0.0f;  // F32P64: offsets from the slice centre
    if (LIK) {
        const double f0 = floor((t0 - a.bc0) * a.lik_inv_w);
        const double f1 = floor((t1 - a.bc0) * a.lik_inv_w);
        in0 = f0 >= 0.0 && f0 < (double)(a.S - 1);
        in1 = f1 >= 0.0 && f1 < (double)(a.S - 1);
        const int k0 = in0 ? (int)f0 : 0, k1 = in1 ? (int)f1 : 0;
        tb0 = __ldg(reinterpret_cast<const TB*>(a.table) + k0);
        tb1 = __ldg(reinterpret_cast<const TB*>(a.table) + k1);
        if (PREC == PREC_F32P64) {
            // offsets from the slice centre, needed before t changes
            x0f = (float)(t0 - (a.bc0 + (double)k0 * a.bw));
            x1f = (float)(t1 - (a.bc0 + (double)k1 * a.bw));
        }
    }
    E s0, s1;
    if (PREC == PREC_F64) {
        double x0 = 0.0, x1 = 0.0;
        for (int j = 0; j < a.n_rf; ++j) {
            x0 += c.V[j] * sin(c.om[j] * t0 + c.ph[j]);
            x1 += c.V[j] * sin(c.om[j] * t1 + c.ph[j]);
        }
        s0 = (E)x0;
        s1 = (E)x1;
    } else {
        float x0 = 0.0f, x1 = 0.0f;
        for (int j = 0; j < a.n_rf; ++j) {
            x0 += c.Vf[j] * sinf((float)reduce_2pi(fma(c.om[j], t0, c.ph[j])));
            x1 += c.Vf[j] * sinf((float)reduce_2pi(fma(c.om[j], t1, c.ph[j])));
        }
        s0 = (E)x0;
        s1 = (E)x1;
    }
    if (LIK) {
        if (PREC == PREC_F64) {
            if (in0) e0 += t0 * tb0.x + tb0.y;
            if (in1) e1 += t1 * tb1.x + tb1.y;
        } else {
            if (in0) e0 += __fmaf_rn(tb0.y, x0f, tb0.x);
            if (in1) e1 += __fmaf_rn(tb1.y, x1f, tb1.x);
        }
    }
    const E q = (E)a.charge, acc = (E)c.acc;
    e0 += q * s0 + acc;
    e1 += q * s1 + acc;
    if (SOLVER == BLOND_SOLVER_SIMPLE) {
        t0 = drift_simple<double>(t0, (double)e0, c.d.simple);
        t1 = drift_simple<double>(t1, (double)e1, c.d.simple);
    } else if (SOLVER == BLOND_SOLVER_LEGACY) {
        t0 = drift_legacy<double>(t0, (double)e0, c.d.Tr, c.d.e0, c.d.e1, c.d.e2, order);
        t1 = drift_legacy<double>(t1, (double)e1, c.d.Tr, c.d.e0, c.d.e1, c.d.e2, order);
    } else {
        t0 = drift_exact<double>(t0, (double)e0, c.d.Tr, c.d.ib2, c.d.ie2, c.d.a0, c.d.a1,
                                 c.d.a2, c.d.energy);
        t1 = drift_exact<double>(t1, (double)e1, c.d.Tr, c.d.ib2, c.d.ie2, c.d.a0, c.d.a1,
                                 c.d.a2, c.d.energy);
    }
}

__device__ __forceinline__ int engine_bin(double t, double cut_left, double inv_w, int S) {
    const double f = floor(__dmul_rn(__dsub_rn(t, cut_left), inv_w));
    return (f >= 0.0 && f < (double)S) ? (int)f : -1;
}

__device__ __forceinline__ void deposit(int* sh, int b, bool warp_agg, unsigned mask) {
    if (warp_agg) {
        const unsigned peers = __match_any_sync(mask, b);
        if (b >= 0 && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&sh[b], __popc(peers));
    } else if (b >= 0) {
        atomicAdd(&sh[b], 1);
    }
}

// Block-private histogram layouts of the staged particle pass.
//   HIST_AGG    one int per bin, warp-aggregated deposits (short profiles)
//   HIST_I32    one int per bin
//   HIST_PACKED two 16-bit counters per 32-bit word -- bin b < half in the
//               low half of word b, bin b >= half in the high half of word
//               b - half -- so a 2^16-slice profile fits in 128 KB.
enum { HIST_AGG = 0, HIST_I32 = 1, HIST_PACKED = 2 };

// Packed deposit.  A counter wraps after 65536 deposits of one block into
// one bin; every wrap is seen by exactly one thread (from the old value its
// atomic returns) and carried into the global histogram, so the counts stay
// exact for any distribution.  A low counter's wrap also carries +1 into
// the high counter of the word; the depositing thread takes that carry
// back, and both the carry and its removal may wrap the high counter, which
// is accounted the same way.  Between the carry and its removal the high
// counter only ever holds extra carries (never fewer), so the accounting
// needs no ordering between threads.
__device__ __forceinline__ void deposit_packed(unsigned* sh, int half, int* gh, int b) {
    if (b < 0) return;
    if (b < half) {
        const unsigned old = atomicAdd(&sh[b], 1u);
        if ((old & 0xffffu) == 0xffffu) {
            atomicAdd(&gh[b], 65536);
            if ((old >> 16) == 0xffffu) atomicAdd(&gh[b + half], 65536);
            const unsigned o2 = atomicSub(&sh[b], 0x10000u);
            if ((o2 >> 16) == 0u) atomicAdd(&gh[b + half], -65536);
        }
    } else {
        const unsigned old = atomicAdd(&sh[b - half], 0x10000u);
        if ((old >> 16) == 0xffffu) atomicAdd(&gh[b], 65536);
    }
}

template <int HIST>
__device__ __forceinline__ void block_deposit(int* sh, int half, int* gh, int b) {
    if (HIST == HIST_PACKED)
        deposit_packed(reinterpret_cast<unsigned*>(sh), half, gh, b);
    else
        deposit(sh, b, HIST == HIST_AGG, 0xffffffffu);
}

// Flush the block-private histograms of one thread-block cluster: CTA r sums
// bin range r of every CTA's shared histogram through distributed shared
// memory and adds the sums to the global histogram, so a cluster of C
// blocks issues S global atomics instead of C * S.  (A launch without a
// cluster attribute is a cluster of one.)
__device__ __forceinline__ void cluster_flush(int* sh, int* hist, int S) {
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const int C = (int)cl.num_blocks();
    const int r = (int)cl.block_rank();
    cl.sync();  // every CTA of the cluster has finished depositing
    const int per = (S + C - 1) / C;
    const int hi = min(S, (r + 1) * per);
    for (int k = r * per + threadIdx.x; k < hi; k += blockDim.x) {
        int sum = 0;
        for (int q = 0; q < C; ++q) sum += cl.map_shared_rank(sh, q)[k];
        if (sum) atomicAdd(&hist[k], sum);
    }
    cl.sync();  // remote reads done before any CTA's shared memory goes away
}

// Largest block of the plain pass; its launch bound (1024 threads, one
// block per SM) caps registers at 64 per thread, the same as two blocks of
// 512, so 256-, 512- and 1024-thread launches all use the same code.
constexpr int kEngineThreads = 1024;

// The particle arrays stream through L2 once per turn (hundreds of MB
// against a 126 MB L2).  Their loads and stores carry an L2 evict-first
// policy, so they are the lines replaced first and the head kernel's code,
// twiddles, impedance and the interpolation table stay in L2 from one turn
// to the next (C2, FP64: 99.8 -> 94.2 us per turn, the head 30.5 -> 27 us).
__device__ __forceinline__ uint64_t evict_first_policy() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
// Per-thread asynchronous copies into shared memory (cp.async, 16 or 8
// bytes): the prefetch ring of the plain pass.
__device__ __forceinline__ void ring_copy16(void* smem, const void* gmem, uint64_t pol) {
    asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(smem)), "l"(gmem), "l"(pol) : "memory");
}
__device__ __forceinline__ void ring_copy8(void* smem, const void* gmem, uint64_t pol) {
    asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 8, %2;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(smem)), "l"(gmem), "l"(pol) : "memory");
}
__device__ __forceinline__ void stream_store(double2* p, double2 v, uint64_t pol) {
    asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(p), "d"(v.x),
                 "d"(v.y), "l"(pol) : "memory");
}
__device__ __forceinline__ void stream_store(float2* p, float2 v, uint64_t pol) {
    asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(p), "f"(v.x),
                 "f"(v.y), "l"(pol) : "memory");
}
__device__ __forceinline__ void stream_store(double* p, double v, uint64_t pol) {
    asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(p), "d"(v), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void stream_store(float* p, float v, uint64_t pol) {
    asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(v), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ double2 stream_load(const double2* p, uint64_t pol) {
    double2 v;
    asm volatile("ld.global.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
                 : "=d"(v.x), "=d"(v.y) : "l"(p), "l"(pol) : "memory");
    return v;
}
__device__ __forceinline__ float2 stream_load(const float2* p, uint64_t pol) {
    float2 v;
    asm volatile("ld.global.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;"
                 : "=f"(v.x), "=f"(v.y) : "l"(p), "l"(pol) : "memory");
    return v;
}
__device__ __forceinline__ double stream_load(const double* p, uint64_t pol) {
    double v;
    asm volatile("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol)
                 : "memory");
    return v;
}
__device__ __forceinline__ float stream_load(const float* p, uint64_t pol) {
    float v;
    asm volatile("ld.global.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol)
                 : "memory");
    return v;
}
// Bulk prefetch of a byte range into L2 (no completion to wait for).
__device__ __forceinline__ void l2_prefetch(const void* p, uint32_t bytes, uint64_t pol) {
    asm volatile("cp.async.bulk.prefetch.L2.global.L2::cache_hint [%0], %1, %2;" ::"l"(p),
                 "r"(bytes), "l"(pol) : "memory");
}
// The 16-byte aligned part of [lo, hi) into L2.
__device__ __forceinline__ void l2_prefetch_range(const void* lo, const void* hi, uint64_t pol) {
    const uintptr_t a = ((uintptr_t)lo + 15) & ~(uintptr_t)15, b = (uintptr_t)hi & ~(uintptr_t)15;
    if (b > a) l2_prefetch(reinterpret_cast<const void*>(a), (uint32_t)(b - a), pol);
}
__device__ __forceinline__ void ring_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void ring_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Bytes of the plain pass's prefetch ring per thread and stage.
template <int PREC>
constexpr int ring_bytes() {
    return 16 + (PREC == PREC_F64 ? 16 : 8);
}

// Pairs of particles per thread and iteration; pairs are read with one
// 16-byte (dt) and one 16- or 8-byte (dE) load.  With NST > 0 the loads go
// through a per-thread ring of NST shared-memory slots filled NST - 1
// iterations ahead with cp.async: each thread then has NST - 1 pairs in
// flight while it computes one, without extra registers and without any
// block-wide barrier (a thread reads only the slots it filled itself).
template <int PREC, int SOLVER, bool LIK, bool KICK, bool WARP_AGG, int NST>
__global__ void __launch_bounds__(kEngineThreads, 1)
particle_kernel(const ParticleArgs a) {
    using E = typename Coord<PREC>::E;
    using E2 = typename Vec2<E>::type;
    extern __shared__ __align__(16) int sh[];
    __shared__ TurnConsts c;
    // launched with programmatic serialization (the engine's turn): the
    // next turn's head may launch now and set itself up; this block clears
    // its histogram, then waits for the head (turn counter, RF programme,
    // table, cleared global histogram) before reading anything it wrote
    pdl_launch_dependents();
    // profiles too long for a shared-memory copy deposit straight into
    // the global histogram
    int* const hd = a.global_hist ? a.hist : sh;
    if (!a.global_hist)
        for (int k = threadIdx.x; k < a.S; k += blockDim.x) sh[k] = 0;
    pdl_wait();
    long long t_idx = a.turn ? (*a.turn - 1) : 0;
    if (t_idx < 0) t_idx = 0;
    if (t_idx >= a.n_turns) t_idx = a.n_turns - 1;
    if (KICK) {
        for (int j = threadIdx.x; j < a.n_rf; j += blockDim.x) {
            c.V[j] = a.V[t_idx * a.n_rf + j];
            c.Vf[j] = (float)c.V[j];
            c.om[j] = a.om[t_idx * a.n_rf + j];
            c.ph[j] = a.ph[t_idx * a.n_rf + j];
        }
        if (threadIdx.x == 0) {
            c.acc = a.acc[t_idx];
            c.d = a.drift[t_idx + 1];
        }
    }
    __syncthreads();

    double* dt = reinterpret_cast<double*>(a.dt);
    E* dE = reinterpret_cast<E*>(a.dE);
    const int64_t npairs = a.n / 2;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int order = a.order;
    // whole warps iterate together (needed by __match_any_sync)
    const int lane = threadIdx.x & 31;
    int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31);
    const uint64_t pol = evict_first_policy();
    if (NST == 0) {
        for (; base < npairs; base += stride) {
            const int64_t p = base + lane;
            int b0 = -1, b1 = -1;
            if (p < npairs) {
                double2 tt = stream_load(reinterpret_cast<const double2*>(dt) + p, pol);
                E2 ee = stream_load(reinterpret_cast<const E2*>(dE) + p, pol);
                if (KICK) track_pair<PREC, SOLVER, LIK>(tt.x, tt.y, ee.x, ee.y, c, a, order);
                if (KICK) {
                    stream_store(reinterpret_cast<double2*>(dt) + p, tt, pol);
                    stream_store(reinterpret_cast<E2*>(dE) + p, ee, pol);
                }
                b0 = engine_bin(tt.x, a.cut_left, a.inv_w, a.S);
                b1 = engine_bin(tt.y, a.cut_left, a.inv_w, a.S);
            }
            deposit(hd, b0, WARP_AGG, 0xffffffffu);
            deposit(hd, b1, WARP_AGG, 0xffffffffu);
        }
    } else {
        // the ring sits after the (16-byte aligned) histogram
        const size_t hbytes = a.global_hist ? 0 : (((size_t)a.S * sizeof(int) + 15) & ~(size_t)15);
        double2* rdt = reinterpret_cast<double2*>(reinterpret_cast<char*>(sh) + hbytes);
        E2* rdE = reinterpret_cast<E2*>(rdt + (size_t)NST * blockDim.x);
        const double2* gdt = reinterpret_cast<const double2*>(dt);
        const E2* gdE = reinterpret_cast<const E2*>(dE);
        auto fill = [&](int slot, int64_t p) {
            if (p < npairs) {
                ring_copy16(&rdt[slot * blockDim.x + threadIdx.x], &gdt[p], pol);
                if (sizeof(E2) == 16) ring_copy16(&rdE[slot * blockDim.x + threadIdx.x], &gdE[p], pol);
                else ring_copy8(&rdE[slot * blockDim.x + threadIdx.x], &gdE[p], pol);
            }
            ring_commit();  // one group per stage, empty past the end
        };
#pragma unroll
        for (int s = 0; s < NST - 1; ++s) fill(s, base + s * stride + lane);
        int slot = 0;
        for (; base < npairs; base += stride) {
            // stage it + NST - 1 goes into the slot this thread emptied in
            // the previous iteration
            fill(slot == 0 ? NST - 1 : slot - 1, base + (NST - 1) * stride + lane);
            // F32P64: thread 0 also prefetches into L2 the block's slice one
            // iteration beyond the ring, so each SM has twice the bytes in
            // flight without more shared memory (C2: particle pass 58.4 ->
            // 54.0 us; FP64 lost ~2 us a turn with it, so it is F32P64 only)
            if (PREC == PREC_F32P64 && threadIdx.x == 0) {
                const int64_t pb = base + (int64_t)NST * stride;
                if (pb < npairs) {
                    const int64_t cnt = min((int64_t)blockDim.x, npairs - pb);
                    if (((uintptr_t)(gdt + pb) & 15) == 0)
                        l2_prefetch(gdt + pb, (uint32_t)(cnt * 16), pol);
                    if (((uintptr_t)(gdE + pb) & 15) == 0 && ((cnt * sizeof(E2)) & ~(int64_t)15))
                        l2_prefetch(gdE + pb, (uint32_t)((cnt * sizeof(E2)) & ~(int64_t)15), pol);
                }
            }
            ring_wait<NST - 1>();  // groups complete in order: this stage landed
            const int64_t p = base + lane;
            int b0 = -1, b1 = -1;
            if (p < npairs) {
                double2 tt = rdt[slot * blockDim.x + threadIdx.x];
                E2 ee = rdE[slot * blockDim.x + threadIdx.x];
                track_pair<PREC, SOLVER, LIK>(tt.x, tt.y, ee.x, ee.y, c, a, order);
                stream_store(reinterpret_cast<double2*>(dt) + p, tt, pol);
                stream_store(reinterpret_cast<E2*>(dE) + p, ee, pol);
                b0 = engine_bin(tt.x, a.cut_left, a.inv_w, a.S);
                b1 = engine_bin(tt.y, a.cut_left, a.inv_w, a.S);
            }
            deposit(hd, b0, WARP_AGG, 0xffffffffu);
            deposit(hd, b1, WARP_AGG, 0xffffffffu);
            slot = slot + 1 == NST ? 0 : slot + 1;
        }
        ring_wait<0>();  // nothing may land in shared memory after the flush
    }
    // odd tail particle
    if ((a.n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        double t = dt[a.n - 1];
        E e = dE[a.n - 1];
        track_one<PREC, SOLVER, LIK, KICK, true, false>(t, e, c, a, sh, order);
        if (KICK) {
            dt[a.n - 1] = t;
            dE[a.n - 1] = e;
        }
        const int b = engine_bin(t, a.cut_left, a.inv_w, a.S);
        if (b >= 0) atomicAdd(&hd[b], 1);
    }
    if (!a.global_hist) cluster_flush(sh, a.hist, a.S);
}

// ------------------------------------------------------ TMA-pipelined pass
// The plain kernel above is latency-bound (ncu: long-scoreboard stalls at
// 50% occupancy): each warp has only its own few loads in flight while it
// computes the FP64 sines.  Here one block per SM streams fixed-size chunks
// of dt/dE into shared memory with bulk asynchronous copies
// (cp.async.bulk ... mbarrier::complete_tx) kSt stages ahead, so the copy
// engine keeps the HBM busy while the warps compute; results go straight
// back to global memory with coalesced stores.
constexpr int kTile = 2048;    // particles per chunk
constexpr int kStages = 4;     // chunks in flight per block
constexpr int kTmaThreads = 1024;  // 32 warps: enough to hide the FP64 sine chains
constexpr long long kWaitLimit = 1LL << 26;  // bounded mbarrier spin

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar, uint64_t pol) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint "
        "[%0], [%1], %2, [%3], %4;" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(pol)
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.b32 %0, 1, 0, p;\n}" : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}
// Bounded wait, warp-uniform: every lane polls (each needs the acquire of
// the completed phase) and the warp leaves together.  Returns false (and
// sets the error word) if the copy never lands.
__device__ __forceinline__ bool mbar_wait_warp(uint64_t* bar, uint32_t parity, int* err) {
    for (long long it = 0; it < kWaitLimit; ++it)
        if (__all_sync(0xffffffffu, mbar_try_wait(bar, parity))) return true;
    if ((threadIdx.x & 31) == 0) atomicExch(err, 1);
    return false;
}
// Single-thread bounded wait used on the error path.
__device__ __forceinline__ void mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (long long it = 0; it < kWaitLimit; ++it)
        if (mbar_try_wait(bar, parity)) return;
}

template <int PREC, int SOLVER, bool LIK, int HIST>
__global__ void __launch_bounds__(kTmaThreads, 1)
particle_kernel_tma(const ParticleArgs a, int* err) {
    using E = typename Coord<PREC>::E;
    using E2 = typename Vec2<E>::type;
    extern __shared__ __align__(128) unsigned char dsm[];
    __shared__ TurnConsts c;
    __shared__ __align__(8) uint64_t full[kStages];
    int* sh = reinterpret_cast<int*>(dsm);
    const int half = (a.S + 1) / 2;
    const int words = HIST == HIST_PACKED ? half : a.S;
    const int nst = a.tma_stages;  // 2 .. kStages chunks in flight
    const size_t hist_bytes = ((size_t)words * sizeof(int) + 127) & ~(size_t)127;
    double* st_dt = reinterpret_cast<double*>(dsm + hist_bytes);
    E* st_dE = reinterpret_cast<E*>(dsm + hist_bytes + sizeof(double) * kTile * nst);

    long long t_idx = a.turn ? (*a.turn - 1) : 0;
    if (t_idx < 0) t_idx = 0;
    if (t_idx >= a.n_turns) t_idx = a.n_turns - 1;
    for (int j = threadIdx.x; j < a.n_rf; j += blockDim.x) {
        c.V[j] = a.V[t_idx * a.n_rf + j];
        c.Vf[j] = (float)c.V[j];
        c.om[j] = a.om[t_idx * a.n_rf + j];
        c.ph[j] = a.ph[t_idx * a.n_rf + j];
    }
    if (threadIdx.x == 0) {
        c.acc = a.acc[t_idx];
        c.d = a.drift[t_idx + 1];
        for (int s = 0; s < nst; ++s) mbar_init(&full[s], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int k = threadIdx.x; k < words; k += blockDim.x) sh[k] = 0;
    __syncthreads();

    double* dt = reinterpret_cast<double*>(a.dt);
    E* dE = reinterpret_cast<E*>(a.dE);
    const long long nchunks = a.n / kTile;
    // this block's chunks: blockIdx.x, blockIdx.x + gridDim.x, ...
    const long long mine = nchunks > blockIdx.x
                               ? (nchunks - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const uint32_t bytes_dt = sizeof(double) * kTile, bytes_dE = sizeof(E) * kTile;
    const uint64_t pol = evict_first_policy();
    auto issue = [&](long long i) {
        const int s = (int)(i % nst);
        const long long chunk = blockIdx.x + i * gridDim.x;
        mbar_expect_tx(&full[s], bytes_dt + bytes_dE);
        bulk_g2s(st_dt + (size_t)s * kTile, dt + chunk * kTile, bytes_dt, &full[s], pol);
        bulk_g2s(st_dE + (size_t)s * kTile, dE + chunk * kTile, bytes_dE, &full[s], pol);
    };
    if (threadIdx.x == 0)
        for (long long i = 0; i < mine && i < nst; ++i) issue(i);

    const int order = a.order;
    for (long long i = 0; i < mine; ++i) {
        const int s = (int)(i % nst);
        const bool got = mbar_wait_warp(&full[s], (uint32_t)((i / nst) & 1), err);
        if (got) {
            const long long base = (blockIdx.x + i * gridDim.x) * (long long)kTile;
            const double2* sdt = reinterpret_cast<const double2*>(st_dt + (size_t)s * kTile);
            const E2* sdE = reinterpret_cast<const E2*>(st_dE + (size_t)s * kTile);
#pragma unroll
            for (int q = 0; q < kTile / 2 / kTmaThreads; ++q) {
                const int p = threadIdx.x + q * kTmaThreads;  // pair within the chunk
                double2 tt = sdt[p];
                E2 ee = sdE[p];
                track_pair<PREC, SOLVER, LIK>(tt.x, tt.y, ee.x, ee.y, c, a, order);
                stream_store(reinterpret_cast<double2*>(dt + base) + p, tt, pol);
                stream_store(reinterpret_cast<E2*>(dE + base) + p, ee, pol);
                block_deposit<HIST>(sh, half, a.hist, engine_bin(tt.x, a.cut_left, a.inv_w, a.S));
                block_deposit<HIST>(sh, half, a.hist, engine_bin(tt.y, a.cut_left, a.inv_w, a.S));
            }
        }
        // stage s fully consumed; the failure decision is block-uniform
        if (__syncthreads_or(!got)) {
            // copies i .. min(mine, i + nst) - 1 are in flight: give
            // them a bounded chance to land before the block's shared
            // memory is released, then leave without flushing
            if (threadIdx.x == 0)
                for (long long j = i; j < mine && j < i + nst; ++j)
                    mbar_wait_bounded(&full[j % nst], (uint32_t)((j / nst) & 1));
            __syncthreads();
            return;
        }
        if (threadIdx.x == 0 && i + nst < mine) {
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue(i + nst);
        }
    }
    // remainder particles (fewer than one chunk): plain loads, last block
    if (blockIdx.x == gridDim.x - 1) {
        for (long long i = nchunks * kTile + threadIdx.x; i < a.n; i += blockDim.x) {
            double t = dt[i];
            E e = dE[i];
            track_one<PREC, SOLVER, LIK, true, true, false>(t, e, c, a, sh, order);
            dt[i] = t;
            dE[i] = e;
            const int b = engine_bin(t, a.cut_left, a.inv_w, a.S);
            if (HIST == HIST_PACKED)
                deposit_packed(reinterpret_cast<unsigned*>(sh), half, a.hist, b);
            else if (b >= 0)
                atomicAdd(&sh[b], 1);
        }
    }
    __syncthreads();
    if (HIST == HIST_PACKED) {
        const unsigned* shp = reinterpret_cast<const unsigned*>(sh);
        for (int k = threadIdx.x; k < half; k += blockDim.x) {
            const unsigned v = shp[k];
            if (v & 0xffffu) atomicAdd(&a.hist[k], (int)(v & 0xffffu));
            if ((v >> 16) && k + half < a.S) atomicAdd(&a.hist[k + half], (int)(v >> 16));
        }
    } else {
        for (int k = threadIdx.x; k < a.S; k += blockDim.x) {
            const int v = sh[k];
            if (v) atomicAdd(&a.hist[k], v);
        }
    }
}

// Profile <- histogram.  With clear, the histogram is zeroed and the turn
// counter advanced (the head of a turn without induced voltage).
__global__ void profile_kernel(int* hist, double* profile, int S, int clear,
                               long long* turn) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < S;
         k += gridDim.x * blockDim.x) {
        profile[k] = (double)hist[k];
        if (clear) hist[k] = 0;
    }
    if (clear && turn && blockIdx.x == 0 && threadIdx.x == 0) *turn += 1;
}

}  // namespace bb

using namespace bb;

struct blond_engine {
    int precision = 0, n_rf = 0, solver = 0, S = 0;
    int device = 0;
    // programme
    int64_t n_turns = 0;
    double charge = 1.0;
    double* d_V = nullptr;
    double* d_om = nullptr;
    double* d_ph = nullptr;
    double* d_acc = nullptr;
    DriftTurn* d_drift = nullptr;
    int order = 0;
    bool rf_set = false, drift_set = false;
    std::vector<double> h_t_rev;
    // slicing
    bool slicing_set = false;
    double cut_left = 0, cut_right = 0, inv_w = 0;
    double* d_bc = nullptr;
    double bc0 = 0, lik_inv_w = 0, bw = 0, dbc = 0;
    // impedance
    bool has_fft = false;
    SpecPlan plan = {};
    double2* d_H = nullptr;
    double2* d_tw = nullptr;  // twiddle tables of the spectral plan
    double iv_scale = 0.0;
    bool has_ind = false;
    double* d_ind = nullptr;
    // beam-phase loop (blond_engine_set_feedback)
    bool has_fb = false;
    bb::FeedbackArgs fb = {};
    double* d_fb_table = nullptr;
    double* d_fb_on_time = nullptr;
    double* d_fb_state = nullptr;
    double* d_fb_trace = nullptr;
    double* d_fb_partials = nullptr;  // dE partials, then the beam-phase partials
    int* d_fb_ticket = nullptr;  // last-block ticket of the loop pass (0 between passes)
    // state
    long long* d_turn = nullptr;
    int* d_err = nullptr;  // set by a kernel whose bounded wait gave up
    long long host_turn = 0;
    int* d_hist = nullptr;    // the histogram in use (own or caller-bound)
    int* own_hist = nullptr;  // the one engine_create allocated
    double* d_profile = nullptr;
    double* d_vind = nullptr;
    void* d_table = nullptr;
    // beam
    void* dt = nullptr;
    void* dE = nullptr;
    int64_t n = 0;
    // tuning
    int threads = 512;
    int blocks_per_sm = 2;
    int turns_per_graph = 50;
    int variant = 0;  // 0: TMA-pipelined particle pass, 1: plain loads
    int hist_mode = -1;  // -1 automatic, else HIST_AGG/I32/PACKED/GLOBAL
    int ring = 0;        // plain pass: prefetch ring stages (0 = direct loads)
    int cluster = 1;     // plain pass: blocks whose histograms merge on chip
    // programmatic dependent launch between the turn's head and particle
    // pass: each kernel lets the next one launch and set up early
    bool pdl = true;
    // host-buffer pipeline (blond_engine_track_host): copy streams and one
    // (in, done, out) event triple per chunk
    cudaStream_t io_in = nullptr, io_out = nullptr;
    std::vector<cudaEvent_t> io_ev;
    // graph cache
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_turns = 0;
    bool graph_dirty = true;
};

namespace bb {

static void free_ptr(void* p) {
    if (p) cudaFree(p);
}

// Largest profile whose histogram the particle kernel privatises in shared
// memory; longer profiles deposit into the global histogram.
static int smem_hist_limit() {
    return (device_info().max_smem_optin - (int)sizeof(TurnConsts) - 1024) / 4;
}
static bool global_hist(const blond_engine* e) { return e->S > smem_hist_limit(); }

// Histogram layout of the plain pass: straight into global memory when
// asked for or when one int per bin does not fit in shared memory, else
// block-private, warp-aggregated when asked for or for short profiles.
enum { HIST_GLOBAL = 3 };
static bool plain_global(const blond_engine* e) {
    return global_hist(e) || e->hist_mode == HIST_GLOBAL;
}
static bool plain_agg(const blond_engine* e) {
    if (e->hist_mode == HIST_AGG) return true;
    if (e->hist_mode == HIST_I32) return false;
    return e->S <= 2048;
}
static int engine_smem(const blond_engine* e) {
    return plain_global(e) ? 0 : (int)sizeof(int) * e->S;
}

// Raise a kernel's dynamic shared memory limit to the device's opt-in
// maximum, once per device.  Done outside stream capture (engine_run calls
// the launchers with launch=false before it captures).
template <typename K>
static int allow_max_smem(K kernel, bool* done) {
    const DeviceInfo& d = device_info();
    if (!done[d.device & 63]) {
        // the opt-in limit covers static + dynamic shared memory
        cudaFuncAttributes fa;
        BB_CUDA(cudaFuncGetAttributes(&fa, kernel));
        BB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     d.max_smem_optin - (int)fa.sharedSizeBytes));
        done[d.device & 63] = true;
    }
    return BLOND_OK;
}

// Layout of the staged pass for a profile of S slices: the histogram mode
// and the number of chunks in flight that fit beside it in shared memory
// (0: not even two fit, the plain pass runs instead).  One int per bin is
// kept while it leaves room for kStages chunks (or as many as the packed
// layout would); beyond that the packed 16-bit layout halves the
// histogram.
struct TmaPlan {
    int mode = HIST_I32;
    int stages = 0;
    size_t bytes = 0;
};

template <int PREC>
static TmaPlan tma_plan(int S, int forced) {
    using E = typename Coord<PREC>::E;
    const size_t stage = (size_t)kTile * (sizeof(double) + sizeof(E));
    // static shared memory of the kernel (TurnConsts, barriers) + margin
    const size_t reserve = sizeof(TurnConsts) + sizeof(uint64_t) * kStages + 256;
    const size_t limit = (size_t)device_info().max_smem_optin - reserve;
    auto fit = [&](size_t words, int* st) {
        const size_t hist = (words * sizeof(int) + 127) & ~(size_t)127;
        *st = hist + 2 * stage > limit
                  ? 0 : (int)std::min<size_t>(kStages, (limit - hist) / stage);
        return hist;
    };
    int st_i = 0, st_p = 0;
    const size_t h_i = fit((size_t)S, &st_i);
    const size_t h_p = fit((size_t)(S + 1) / 2, &st_p);
    TmaPlan p;
    if (forced == HIST_GLOBAL) return p;
    if (forced == HIST_AGG || forced == HIST_I32) {
        if (st_i >= 2) {
            p.mode = forced;
            p.stages = st_i;
            p.bytes = h_i + (size_t)st_i * stage;
        }
        return p;
    }
    if (forced == HIST_PACKED) {
        if (st_p >= 2) {
            p.mode = HIST_PACKED;
            p.stages = st_p;
            p.bytes = h_p + (size_t)st_p * stage;
        }
        return p;
    }
    if (st_i >= 2 && st_i >= std::min(kStages, st_p)) {
        p.mode = S <= 2048 ? HIST_AGG : HIST_I32;
        p.stages = st_i;
        p.bytes = h_i + (size_t)st_i * stage;
    } else if (st_p >= 2) {
        p.mode = HIST_PACKED;
        p.stages = st_p;
        p.bytes = h_p + (size_t)st_p * stage;
    }
    return p;
}

template <int PREC, int SOLVER, bool LIK, int HIST>
static int launch_tma(blond_engine* e, ParticleArgs a, const TmaPlan& p, cudaStream_t s,
                      bool launch) {
    static bool done[64] = {false};
    auto k = particle_kernel_tma<PREC, SOLVER, LIK, HIST>;
    int rc;
    if ((rc = allow_max_smem(k, done))) return rc;
    a.tma_stages = p.stages;
    const long long nchunks = a.n / kTile;
    const int grid = (int)std::max<long long>(
        1, std::min<long long>(nchunks, device_info().sm_count));
    if (launch) k<<<grid, kTmaThreads, p.bytes, s>>>(a, e->d_err);
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

// Raise a kernel's dynamic shared memory limit to the opt-in maximum once
// per (kernel, device).
template <typename K>
static int allow_smem_once(K kernel) {
    static std::mutex mu;
    static std::set<std::pair<const void*, int>> done;
    const DeviceInfo& d = device_info();
    const std::pair<const void*, int> key(reinterpret_cast<const void*>(kernel), d.device);
    std::lock_guard<std::mutex> lock(mu);
    if (done.count(key)) return BLOND_OK;
    cudaFuncAttributes fa;
    BB_CUDA(cudaFuncGetAttributes(&fa, kernel));
    BB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 d.max_smem_optin - (int)fa.sharedSizeBytes));
    done.insert(key);
    return BLOND_OK;
}

// The plain pass for a histogram mode and prefetch ring depth (0, 2, 4).
template <int PREC, int SOLVER, bool LIK, bool KICK>
static auto plain_kernel(bool agg, int ring)
    -> decltype(&particle_kernel<PREC, SOLVER, LIK, KICK, true, 0>) {
    if constexpr (KICK) {
        if (ring == 2)
            return agg ? particle_kernel<PREC, SOLVER, LIK, KICK, true, 2>
                       : particle_kernel<PREC, SOLVER, LIK, KICK, false, 2>;
        if (ring == 4)
            return agg ? particle_kernel<PREC, SOLVER, LIK, KICK, true, 4>
                       : particle_kernel<PREC, SOLVER, LIK, KICK, false, 4>;
    }
    return agg ? particle_kernel<PREC, SOLVER, LIK, KICK, true, 0>
               : particle_kernel<PREC, SOLVER, LIK, KICK, false, 0>;
}

// Dynamic shared memory of the plain pass: the histogram (16-byte aligned)
// and the prefetch ring; -1 if that exceeds the opt-in limit.
template <int PREC>
static int plain_ring_smem(const blond_engine* e, int ring) {
    const int h = engine_smem(e);
    const int bytes = ring ? ((h + 15) & ~15) + ring * e->threads * ring_bytes<PREC>() : h;
    const int limit = device_info().max_smem_optin - (int)sizeof(TurnConsts) - 1024;
    return bytes <= limit ? bytes : -1;
}

template <int PREC, int SOLVER, bool LIK, bool KICK>
static int launch_particles_t(blond_engine* e, const ParticleArgs& a, cudaStream_t s,
                              bool launch) {
    const int smem = engine_smem(e);
    const bool agg = plain_agg(e);
    int rc;
    if (KICK) {
        // the staged pass when asked for (variant 0 or the packed layout),
        // and by default for profiles whose int histogram does not fit
        // beside the plain pass (packed layout instead of global atomics)
        const TmaPlan p = tma_plan<PREC>(e->S, e->hist_mode);
        const bool want = e->variant == 0 || e->hist_mode == HIST_PACKED ||
                          (e->hist_mode < 0 && global_hist(e));
        if (p.stages && want) {
            switch (p.mode) {
                case HIST_AGG: return launch_tma<PREC, SOLVER, LIK, HIST_AGG>(e, a, p, s, launch);
                case HIST_I32: return launch_tma<PREC, SOLVER, LIK, HIST_I32>(e, a, p, s, launch);
                default: return launch_tma<PREC, SOLVER, LIK, HIST_PACKED>(e, a, p, s, launch);
            }
        }
        // profile too long for the staged copy: plain loads below
    }
    int grid = particle_grid(a.n / 2 + 1, e->threads, e->blocks_per_sm);
    const int cl = plain_global(e) ? 1 : e->cluster;  // merging needs shared histograms
    grid = (grid + cl - 1) / cl * cl;
    const int ring = KICK ? e->ring : 0;
    auto k = plain_kernel<PREC, SOLVER, LIK, KICK>(agg, ring);
    if ((rc = allow_smem_once(k))) return rc;
    const int smem_ring = plain_ring_smem<PREC>(e, ring);
    if (smem_ring < 0) {
        set_error("engine: prefetch ring of %d stages does not fit beside the histogram", ring);
        return BLOND_ERR_SIZE;
    }
    if (launch) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(grid, 1, 1);
        cfg.blockDim = dim3(e->threads, 1, 1);
        cfg.dynamicSmemBytes = smem_ring;
        cfg.stream = s;
        cudaLaunchAttribute attr[2];
        int na = 0;
        if (cl > 1) {
            attr[na].id = cudaLaunchAttributeClusterDimension;
            attr[na].val.clusterDim.x = cl;
            attr[na].val.clusterDim.y = 1;
            attr[na].val.clusterDim.z = 1;
            ++na;
        }
        if (e->pdl) {
            attr[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            attr[na].val.programmaticStreamSerializationAllowed = 1;
            ++na;
        }
        cfg.attrs = attr;
        cfg.numAttrs = na;
        BB_CUDA(cudaLaunchKernelEx(&cfg, k, a));
    }
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

template <int PREC>
static int launch_particles_p(blond_engine* e, const ParticleArgs& a, bool kick,
                              cudaStream_t s, bool launch) {
    if (!kick) return launch_particles_t<PREC, 0, false, false>(e, a, s, launch);
    const bool lik = e->has_fft || e->has_ind;
    switch (e->solver) {
        case 0:
            return lik ? launch_particles_t<PREC, 0, true, true>(e, a, s, launch)
                       : launch_particles_t<PREC, 0, false, true>(e, a, s, launch);
        case 1:
            return lik ? launch_particles_t<PREC, 1, true, true>(e, a, s, launch)
                       : launch_particles_t<PREC, 1, false, true>(e, a, s, launch);
        default:
            return lik ? launch_particles_t<PREC, 2, true, true>(e, a, s, launch)
                       : launch_particles_t<PREC, 2, false, true>(e, a, s, launch);
    }
}

static ParticleArgs particle_args(blond_engine* e) {
    ParticleArgs a = {};
    a.dt = e->dt;
    a.dE = e->dE;
    a.n = e->n;
    a.n_rf = e->n_rf;
    a.charge = e->charge;
    a.V = e->d_V;
    a.om = e->d_om;
    a.ph = e->d_ph;
    a.acc = e->d_acc;
    a.drift = e->d_drift;
    a.order = e->order;
    a.n_turns = e->n_turns;
    a.turn = e->d_turn;
    a.S = e->S;
    a.cut_left = e->cut_left;
    a.inv_w = e->inv_w;
    a.hist = e->d_hist;
    a.table = e->d_table;
    a.bc0 = e->bc0;
    a.lik_inv_w = e->lik_inv_w;
    a.bw = e->bw;
    a.global_hist = plain_global(e) ? 1 : 0;
    return a;
}

static int launch_particles(blond_engine* e, bool kick, cudaStream_t s,
                            bool launch = true) {
    const ParticleArgs a = particle_args(e);
    if (e->precision == BLOND_PREC_F64)
        return launch_particles_p<PREC_F64>(e, a, kick, s, launch);
    return launch_particles_p<PREC_F32P64>(e, a, kick, s, launch);
}

// The particle pass over particles [off, off + cnt) of the bound beam (off
// even, so pairs stay 16-byte aligned); deposits into the same histogram.
static int launch_particles_range(blond_engine* e, int64_t off, int64_t cnt,
                                  cudaStream_t s) {
    ParticleArgs a = particle_args(e);
    const size_t esz = e->precision == BLOND_PREC_F64 ? sizeof(double) : sizeof(float);
    a.dt = static_cast<double*>(e->dt) + off;
    a.dE = static_cast<char*>(e->dE) + esz * (size_t)off;
    a.n = cnt;
    if (e->precision == BLOND_PREC_F64)
        return launch_particles_p<PREC_F64>(e, a, true, s, true);
    return launch_particles_p<PREC_F32P64>(e, a, true, s, true);
}

static int launch_profile(blond_engine* e, bool clear, cudaStream_t s) {
    const int threads = 256;
    const int grid = std::min(64, (e->S + threads - 1) / threads);
    profile_kernel<<<grid, threads, 0, s>>>(e->d_hist, e->d_profile, e->S, clear ? 1 : 0,
                                            clear ? e->d_turn : nullptr);
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

// The beam-phase loop's arguments for this engine's buffers.
static FeedbackArgs fb_args(const blond_engine* e) {
    FeedbackArgs a = e->fb;
    a.turn = e->d_turn;
    a.profile = e->d_profile;
    a.bc = e->d_bc;
    a.S = e->S;
    a.dt = static_cast<const double*>(e->dt);
    a.dE = e->dE;
    a.dE_f32 = e->precision == BLOND_PREC_F32P64;
    a.n = e->n;
    a.om = e->d_om;
    a.ph = e->d_ph;
    a.table = e->d_fb_table;
    a.on_time = e->d_fb_on_time;
    a.state = e->d_fb_state;
    a.trace = e->d_fb_trace;
    a.partials = e->d_fb_partials;
    a.phase_partials = e->d_fb_partials + kFbPartials;
    a.n_rf = e->n_rf;
    a.n_turns = e->n_turns;
    return a;
}

static int launch_spectral_head(blond_engine* e, cudaStream_t s, bool loop);

// The head of a turn: profile (and induced voltage, table).  With a
// beam-phase loop the spectral head also forms the beam-phase sums while it
// converts the histogram, and its last CTA runs the loop (it corrects the
// next turn's RF programme); without a spectral head one all-SM pass does
// the conversion and the loop.  SPS_RL first sums dE over the beam.
static int launch_head(blond_engine* e, cudaStream_t s) {
    int rc;
    if (!e->has_fb) return launch_spectral_head(e, s, false);
    const FeedbackArgs a = fb_args(e);
    if (!e->has_fft) {
        if ((rc = launch_feedback_dE(a, s))) return rc;
        return launch_feedback_turn(a, e->d_hist, e->d_fb_ticket, 1, s);
    }
    if (a.machine != BLOND_FB_SPS_RL) return launch_spectral_head(e, s, true);
    // SPS_RL averages dE after the induced-voltage kick (the reference's
    // TotalInducedVoltage.track precedes RingAndRFTracker.track): head
    // first, then that average, then the loop on the head's profile
    if ((rc = launch_spectral_head(e, s, false))) return rc;
    if ((rc = launch_feedback_dE_lik(a, e->d_table, e->bc0, e->lik_inv_w, e->bw, s))) return rc;
    return launch_feedback_turn(a, nullptr, e->d_fb_ticket, 0, s);
}

static int launch_spectral_head(blond_engine* e, cudaStream_t s, bool loop) {
    if (!(e->has_fft || e->has_ind)) return launch_profile(e, true, s);
    if (!e->has_fft) {
        set_error("engine: an inductive impedance needs an FFT impedance in this build");
        return BLOND_ERR_UNSUPPORTED;
    }
    SpecParams P = {};
    P.p = e->plan;
    P.mode = SPEC_FORWARD | SPEC_MULTIPLY | SPEC_INVERSE;
    P.pdl = e->pdl ? 1 : 0;
    P.in_i32 = e->d_hist;
    P.n_in = e->S;
    P.profile_out = e->d_profile;
    P.H = e->d_H;
    P.out = e->d_vind;
    P.n_out = std::min<int64_t>(e->S, e->plan.N);
    P.out_scale = -e->iv_scale / (double)e->plan.M;
    P.ind_coeff = e->has_ind ? e->d_ind : nullptr;
    P.ind_dbc = e->dbc;
    P.table = e->d_table;
    P.table_f32 = e->precision == BLOND_PREC_F32P64;
    P.charge = e->charge;
    P.inv_w = e->lik_inv_w;
    P.bc = e->d_bc;
    P.turn = e->d_turn;
    P.bump_turn = 1;
    P.twg = e->d_tw;
    if (loop) {
        SpecLoop L;
        L.ticket = e->d_fb_ticket;
        L.fb = fb_args(e);
        return launch_spectral_loop(P, L, s);
    }
    return launch_spectral(P, s);
}

static int launch_turn(blond_engine* e, cudaStream_t s) {
    int rc = launch_head(e, s);
    if (rc) return rc;
    return launch_particles(e, true, s);
}

static int check_ready(blond_engine* e) {
    if (!e->rf_set || !e->drift_set || !e->slicing_set || !e->dt) {
        set_error("engine: set_rf, set_drift, set_slicing and bind_beam must all be "
                  "called before tracking");
        return BLOND_ERR_STATE;
    }
    return BLOND_OK;
}

static int upload(void** dst, const void* src, size_t bytes) {
    free_ptr(*dst);
    *dst = nullptr;
    BB_CUDA(cudaMalloc(dst, bytes));
    BB_CUDA(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
    return BLOND_OK;
}

}  // namespace bb

extern "C" {

int blond_engine_create(blond_engine** out, int precision, int n_rf, int solver,
                        int n_slices) {
    BB_CHECK_ARG(out, "engine_create: null output");
    BB_CHECK_ARG(precision == BLOND_PREC_F64 || precision == BLOND_PREC_F32P64,
                 "engine_create: unknown precision %d", precision);
    BB_CHECK_SIZE(n_rf >= 1 && n_rf <= kMaxRfEngine, "engine_create: n_rf=%d not in [1, %d]",
                  n_rf, kMaxRfEngine);
    BB_CHECK_ARG(solver >= 0 && solver <= 2, "engine_create: solver %d", solver);
    // beyond smem_hist_limit() slices the histogram lives in global memory
    const int max_s = 1 << 22;
    BB_CHECK_SIZE(n_slices >= 2 && n_slices <= max_s,
                  "engine_create: n_slices=%d not in [2, %d]", n_slices, max_s);
    blond_engine* e = new blond_engine();
    e->precision = precision;
    e->n_rf = n_rf;
    e->solver = solver;
    e->S = n_slices;
    cudaGetDevice(&e->device);
    int rc = BLOND_OK;
    do {
        if (cudaMalloc(&e->d_turn, sizeof(long long)) != cudaSuccess ||
            cudaMalloc(&e->d_err, sizeof(int)) != cudaSuccess ||
            cudaMalloc(&e->d_hist, sizeof(int) * n_slices) != cudaSuccess ||
            cudaMalloc(&e->d_profile, sizeof(double) * n_slices) != cudaSuccess ||
            cudaMalloc(&e->d_vind, sizeof(double) * n_slices) != cudaSuccess ||
            cudaMalloc(&e->d_table, sizeof(double2) * n_slices) != cudaSuccess) {
            set_error("engine_create: cudaMalloc failed");
            rc = BLOND_ERR_CUDA;
            break;
        }
        cudaMemset(e->d_turn, 0, sizeof(long long));
        cudaMemset(e->d_err, 0, sizeof(int));
        cudaMemset(e->d_hist, 0, sizeof(int) * n_slices);
        e->own_hist = e->d_hist;
        cudaMemset(e->d_profile, 0, sizeof(double) * n_slices);
        cudaMemset(e->d_vind, 0, sizeof(double) * n_slices);
        cudaMemset(e->d_table, 0, sizeof(double2) * n_slices);
        if (cudaStreamCreateWithFlags(&e->cap_stream, cudaStreamNonBlocking) != cudaSuccess) {
            set_error("engine_create: stream creation failed");
            rc = BLOND_ERR_CUDA;
            break;
        }
        if (cudaDeviceSynchronize() != cudaSuccess) {
            set_error("engine_create: device error");
            rc = BLOND_ERR_CUDA;
        }
    } while (0);
    if (rc) {
        blond_engine_destroy(e);
        return rc;
    }
    *out = e;
    return BLOND_OK;
}

int blond_engine_destroy(blond_engine* e) {
    if (!e) return BLOND_OK;

    if (e->graph) cudaGraphExecDestroy(e->graph);
    if (e->cap_stream) cudaStreamDestroy(e->cap_stream);
    for (cudaEvent_t ev : e->io_ev) cudaEventDestroy(ev);
    if (e->io_in) cudaStreamDestroy(e->io_in);
    if (e->io_out) cudaStreamDestroy(e->io_out);
    for (void* p : {(void*)e->d_V, (void*)e->d_om, (void*)e->d_ph, (void*)e->d_acc,
                    (void*)e->d_drift, (void*)e->d_bc, (void*)e->d_H, (void*)e->d_tw,
                    (void*)e->d_ind, (void*)e->d_fb_table, (void*)e->d_fb_on_time,
                    (void*)e->d_fb_state, (void*)e->d_fb_trace, (void*)e->d_fb_partials, (void*)e->d_fb_ticket,
                    (void*)e->d_turn, (void*)e->d_err, (void*)e->own_hist, (void*)e->d_profile,
                    (void*)e->d_vind, e->d_table})
        free_ptr(p);
    delete e;
    return BLOND_OK;
}

int blond_engine_set_rf(blond_engine* e, int64_t n_turns, const double* V,
                        const double* om, const double* ph, const double* acc,
                        double charge) {
    BB_CHECK_ARG(e && V && om && ph && acc, "engine_set_rf: null pointer");
    BB_CHECK_ARG(n_turns >= 1, "engine_set_rf: n_turns must be >= 1");
    const size_t cols = (size_t)(n_turns + 1) * e->n_rf;
    int rc;
    if ((rc = upload((void**)&e->d_V, V, sizeof(double) * cols))) return rc;
    if ((rc = upload((void**)&e->d_om, om, sizeof(double) * cols))) return rc;
    if ((rc = upload((void**)&e->d_ph, ph, sizeof(double) * cols))) return rc;
    if ((rc = upload((void**)&e->d_acc, acc, sizeof(double) * n_turns))) return rc;
    e->n_turns = n_turns;
    e->charge = charge;
    e->rf_set = true;
    e->graph_dirty = true;
    return BLOND_OK;
}

int blond_engine_set_drift(blond_engine* e, double length_ratio, double alpha_order,
                           const double* t_rev, const double* eta_0,
                           const double* eta_1, const double* eta_2,
                           const double* alpha_0, const double* alpha_1,
                           const double* alpha_2, const double* beta,
                           const double* energy) {
    BB_CHECK_ARG(e && t_rev && eta_0 && eta_1 && eta_2 && alpha_0 && alpha_1 &&
                     alpha_2 && beta && energy,
                 "engine_set_drift: null pointer");
    BB_CHECK_ARG(e->rf_set, "engine_set_drift: call set_rf first (it fixes n_turns)");
    const int64_t nt = e->n_turns + 1;
    std::vector<DriftTurn> h((size_t)nt);
    e->h_t_rev.assign(t_rev, t_rev + nt);
    for (int64_t i = 0; i < nt; ++i) {
        // drift.cpp:31-56, evaluated once per turn on the host
        DriftTurn d = {};
        d.Tr = t_rev[i] * length_ratio;
        d.simple = d.Tr * eta_0[i] / (beta[i] * beta[i] * energy[i]);
        const double coeff = 1. / (beta[i] * beta[i] * energy[i]);
        d.e0 = eta_0[i] * coeff;
        d.e1 = eta_1[i] * coeff * coeff;
        d.e2 = eta_2[i] * coeff * coeff * coeff;
        d.ib2 = 1 / (beta[i] * beta[i]);
        d.ie2 = 1 / (energy[i] * energy[i]);
        d.energy = energy[i];
        d.a0 = alpha_0[i];
        d.a1 = alpha_1[i];
        d.a2 = alpha_2[i];
        h[(size_t)i] = d;
    }
    e->order = alpha_order == 0 ? 0 : (alpha_order == 1 ? 1 : 2);
    int rc = upload((void**)&e->d_drift, h.data(), sizeof(DriftTurn) * (size_t)nt);
    if (rc) return rc;
    e->drift_set = true;
    e->graph_dirty = true;
    return BLOND_OK;
}

int blond_engine_set_slicing(blond_engine* e, double cut_left, double cut_right,
                             const double* bc) {
    BB_CHECK_ARG(e && bc, "engine_set_slicing: null pointer");
    BB_CHECK_ARG(cut_right > cut_left, "engine_set_slicing: cut_right <= cut_left");
    const int S = e->S;
    e->cut_left = cut_left;
    e->cut_right = cut_right;
    e->inv_w = S / (cut_right - cut_left);  // histogram.cpp:30
    e->bc0 = bc[0];
    e->lik_inv_w = (S - 1) / (bc[S - 1] - bc[0]);  // linear_interp_kick.cpp:31-33
    e->bw = 1.0 / e->lik_inv_w;
    e->dbc = bc[1] - bc[0];
    int rc = upload((void**)&e->d_bc, bc, sizeof(double) * S);
    if (rc) return rc;
    e->slicing_set = true;
    e->graph_dirty = true;
    return BLOND_OK;
}

int blond_engine_set_impedance(blond_engine* e, int64_t n_fft, const double* Z,
                               double scale) {
    BB_CHECK_ARG(e && Z, "engine_set_impedance: null pointer");
    SpecPlan plan;
    if (!make_spec_plan(n_fft, plan)) {
        set_error("engine_set_impedance: n_fft=%lld must be even, 5-smooth and <= %lld",
                  (long long)n_fft, (long long)kMaxClusterFFT);
        return BLOND_ERR_UNSUPPORTED;
    }
    BB_CHECK_SIZE(plan.smem <= device_info().max_smem_optin,
                  "engine_set_impedance: n_fft=%lld needs too much shared memory",
                  (long long)n_fft);
    BB_CHECK_SIZE(n_fft >= e->S, "engine_set_impedance: n_fft=%lld shorter than the "
                  "profile (%d slices)", (long long)n_fft, e->S);
    int rc = upload((void**)&e->d_H, Z, sizeof(double2) * (size_t)(n_fft / 2 + 1));
    if (rc) return rc;
    // twiddle tables of this plan, computed once instead of every turn
    free_ptr(e->d_tw);
    e->d_tw = nullptr;
    if ((rc = make_spec_twiddles(plan, &e->d_tw))) return rc;
    e->plan = plan;
    e->iv_scale = scale;
    e->has_fft = true;
    e->graph_dirty = true;
    return BLOND_OK;
}

int blond_engine_set_inductive(blond_engine* e, const double* z_over_n, double scale) {
    BB_CHECK_ARG(e && z_over_n, "engine_set_inductive: null pointer");
    BB_CHECK_ARG(e->drift_set && e->slicing_set,
                 "engine_set_inductive: call set_drift and set_slicing first");
    // impedance.py:996-1005: -(q e / 2pi) ratio Z/n[t] t_rev[t] / bin_size * grad
    const double bin_size = (e->cut_right - e->cut_left) / e->S;
    std::vector<double> coeff((size_t)e->n_turns + 1);
    for (size_t i = 0; i < coeff.size(); ++i)
        coeff[i] = -(scale * z_over_n[i] * e->h_t_rev[i] / bin_size);
    int rc = upload((void**)&e->d_ind, coeff.data(), sizeof(double) * coeff.size());
    if (rc) return rc;
    e->has_ind = true;
    e->graph_dirty = true;
    return BLOND_OK;
}

int blond_engine_bind_beam(blond_engine* e, void* dt, void* dE, int64_t n) {
    BB_CHECK_ARG(e && dt && dE, "engine_bind_beam: null pointer");
    BB_CHECK_ARG(n >= 1, "engine_bind_beam: n must be >= 1");
    BB_CHECK_ARG(aligned(dt, 16), "engine_bind_beam: dt must be 16-byte aligned");
    // 16 bytes: pair loads, and the bulk copies need 16-byte aligned sources
    BB_CHECK_ARG(aligned(dE, 16), "engine_bind_beam: dE must be 16-byte aligned");
    e->dt = dt;
    e->dE = dE;
    e->n = n;
    e->graph_dirty = true;
    return BLOND_OK;
}

int blond_engine_set_turn(blond_engine* e, int64_t turn, void* stream) {
    BB_CHECK_ARG(e && turn >= 0, "engine_set_turn: bad argument");
    const long long t = turn;
    BB_CUDA(cudaMemcpyAsync(e->d_turn, &t, sizeof(t), cudaMemcpyHostToDevice,
                            as_stream(stream)));
    BB_CUDA(cudaStreamSynchronize(as_stream(stream)));
    e->host_turn = turn;
    return BLOND_OK;
}

int blond_engine_slice(blond_engine* e, void* stream) {
    BB_CHECK_ARG(e, "engine_slice: null engine");
    if (!e->dt || !e->slicing_set) {
        set_error("engine_slice: bind_beam and set_slicing first");
        return BLOND_ERR_STATE;
    }
    cudaStream_t s = as_stream(stream);
    BB_CUDA(cudaMemsetAsync(e->d_hist, 0, sizeof(int) * e->S, s));
    int rc = launch_particles(e, false, s);
    if (rc) return rc;
    return launch_profile(e, false, s);
}

int blond_engine_bind_histogram(blond_engine* e, int* hist) {
    BB_CHECK_ARG(e, "engine_bind_histogram: null engine");
    BB_CHECK_ARG(aligned(hist, 4), "engine_bind_histogram: misaligned histogram");
    e->d_hist = hist ? hist : e->own_hist;
    e->graph_dirty = true;
    return BLOND_OK;
}

int blond_engine_step(blond_engine* e, int part, void* stream) {
    BB_CHECK_ARG(e && part >= 1 && part <= 3, "engine_step: part must be 1, 2 or 3");
    int rc = check_ready(e);
    if (rc) return rc;
    cudaStream_t s = as_stream(stream);
    if (part == 3) return launch_profile(e, false, s);
    BB_CHECK_SIZE(e->host_turn < e->n_turns, "engine_step: turn %lld beyond the programme",
                  (long long)e->host_turn);
    if (part == 1) return launch_head(e, s);
    if ((rc = launch_particles(e, true, s))) return rc;
    e->host_turn += 1;
    return BLOND_OK;
}

int blond_engine_set_kernel(blond_engine* e, int variant) {
    BB_CHECK_ARG(e && (variant == 0 || variant == 1), "engine_set_kernel: variant 0 or 1");
    e->variant = variant;
    e->graph_dirty = true;
    return BLOND_OK;
}

int blond_engine_check(blond_engine* e, void* stream) {
    BB_CHECK_ARG(e, "engine_check: null engine");
    int flag = 0;
    BB_CUDA(cudaMemcpyAsync(&flag, e->d_err, sizeof(int), cudaMemcpyDeviceToHost,
                            as_stream(stream)));
    BB_CUDA(cudaStreamSynchronize(as_stream(stream)));
    if (flag) {
        BB_CUDA(cudaMemsetAsync(e->d_err, 0, sizeof(int), as_stream(stream)));
        set_error("engine: a bounded device-side wait gave up (bulk copy never "
                  "completed); the coordinates of this run are not valid");
        return BLOND_ERR_TIMEOUT;
    }
    return BLOND_OK;
}

int blond_engine_tune(blond_engine* e, int threads, int blocks_per_sm, int turns_per_graph) {
    BB_CHECK_ARG(e, "engine_tune: null engine");
    if (threads) {
        BB_CHECK_ARG(threads % 64 == 0 && threads <= kEngineThreads,
                     "engine_tune: threads must be a multiple of 64 <= %d", kEngineThreads);
        e->threads = threads;
    }
    if (blocks_per_sm) e->blocks_per_sm = blocks_per_sm;
    if (turns_per_graph) e->turns_per_graph = turns_per_graph;
    e->graph_dirty = true;
    return BLOND_OK;
}

int blond_engine_set_cluster(blond_engine* e, int blocks) {
    BB_CHECK_ARG(e && (blocks == 1 || blocks == 2 || blocks == 4 || blocks == 8),
                 "engine_set_cluster: 1, 2, 4 or 8 blocks");
    e->cluster = blocks;
    e->graph_dirty = true;
    return BLOND_OK;
}

int blond_engine_set_prefetch(blond_engine* e, int stages) {
    BB_CHECK_ARG(e && (stages == 0 || stages == 2 || stages == 4),
                 "engine_set_prefetch: stages must be 0, 2 or 4");
    e->ring = stages;
    e->graph_dirty = true;
    return BLOND_OK;
}

int blond_engine_set_histogram(blond_engine* e, int mode) {
    BB_CHECK_ARG(e && mode >= -1 && mode <= HIST_GLOBAL,
                 "engine_set_histogram: mode must be -1 (automatic) .. 3");
    e->hist_mode = mode;
    e->graph_dirty = true;
    return BLOND_OK;
}

// Autotuner of the particle pass.  Every feasible configuration -- plain
// pass with 256 or 512 threads and 1, 2 or 4 blocks per SM (the
// grid-stride loop gives each thread n / (grid x threads) particles),
// each histogram layout and prefetch ring depth (0, 2, 4) that fits, and
// block-private histograms merged in pairs through distributed shared
// memory before the global flush (thread-block clusters of 2);
// staged pass with each layout that fits
// -- is timed on the bound beam with CUDA events (one warm-up and `reps`
// launches each) and the fastest is kept.  The coordinates and the
// histogram are snapshotted first and restored afterwards, so tuning does
// not change the state of the run.
int blond_engine_autotune(blond_engine* e, int reps, void* stream, int* config,
                          double* best_ms) {
    BB_CHECK_ARG(e && config && best_ms && reps >= 1 && reps <= 10,
                 "engine_autotune: bad argument (reps in 1..10)");
    int rc = check_ready(e);
    if (rc) return rc;
    cudaStream_t s = as_stream(stream);
    cudaStreamCaptureStatus cs;
    BB_CUDA(cudaStreamIsCapturing(s, &cs));
    BB_CHECK_ARG(cs == cudaStreamCaptureStatusNone,
                 "engine_autotune: the stream is being captured");
    const size_t esz = e->precision == BLOND_PREC_F64 ? sizeof(double) : sizeof(float);
    const size_t n = (size_t)e->n;
    void *sdt = nullptr, *sdE = nullptr, *shist = nullptr;
    if (cudaMalloc(&sdt, 8 * n) != cudaSuccess || cudaMalloc(&sdE, esz * n) != cudaSuccess ||
        cudaMalloc(&shist, sizeof(int) * (size_t)e->S) != cudaSuccess) {
        free_ptr(sdt);
        free_ptr(sdE);
        free_ptr(shist);
        cudaGetLastError();
        set_error("engine_autotune: cannot allocate the snapshot (%zu bytes)",
                  (8 + esz) * n);
        return BLOND_ERR_CUDA;
    }
    BB_CUDA(cudaMemcpyAsync(sdt, e->dt, 8 * n, cudaMemcpyDeviceToDevice, s));
    BB_CUDA(cudaMemcpyAsync(sdE, e->dE, esz * n, cudaMemcpyDeviceToDevice, s));
    BB_CUDA(cudaMemcpyAsync(shist, e->d_hist, sizeof(int) * e->S, cudaMemcpyDeviceToDevice,
                            s));
    struct Cand { int variant, threads, bps, hist, ring, cluster; };
    std::vector<Cand> cands;
    std::vector<int> plain_modes;
    if (global_hist(e)) plain_modes = {HIST_GLOBAL};
    else if (e->S <= 2048) plain_modes = {HIST_AGG, HIST_I32, HIST_GLOBAL};
    else plain_modes = {HIST_I32, HIST_GLOBAL};
    const bool f64 = e->precision == BLOND_PREC_F64;
    const int keep_threads = e->threads, keep_hist = e->hist_mode;
    for (int threads : {256, 512, 1024})
        for (int bps : {1, 2, 4})
            // 64 registers a thread: at most 1024 threads resident per SM
            if (threads * bps <= 1024)
            for (int h : plain_modes)
                for (int ring : {0, 2, 4})
                    for (int cl : {1, 2}) {
                        if (cl > 1 && (h == HIST_GLOBAL || ring == 4)) continue;
                        e->threads = threads;
                        e->hist_mode = h;
                        const int sm = f64 ? plain_ring_smem<PREC_F64>(e, ring)
                                           : plain_ring_smem<PREC_F32P64>(e, ring);
                        if (sm >= 0) cands.push_back({1, threads, bps, h, ring, cl});
                    }
    e->threads = keep_threads;
    e->hist_mode = keep_hist;
    for (int h : {HIST_AGG, HIST_I32, HIST_PACKED}) {
        if (h == HIST_AGG && e->S > 2048) continue;
        if (h == HIST_I32 && e->S <= 2048) continue;
        const TmaPlan p = f64 ? tma_plan<PREC_F64>(e->S, h) : tma_plan<PREC_F32P64>(e->S, h);
        if (p.stages) cands.push_back({0, kTmaThreads, 1, h, 0, 1});
    }
    const Cand old = {e->variant, e->threads, e->blocks_per_sm, e->hist_mode, e->ring,
                      e->cluster};
    cudaEvent_t a = nullptr, b = nullptr;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    double best = 1e30;
    Cand win = old;
    for (const Cand& c : cands) {
        e->variant = c.variant;
        e->hist_mode = c.hist;
        e->ring = c.ring;
        e->cluster = c.cluster;
        if (c.variant == 1) {
            e->threads = c.threads;
            e->blocks_per_sm = c.bps;
        }
        if (launch_particles(e, true, s, false)) {
            cudaGetLastError();
            continue;
        }
        cudaMemsetAsync(e->d_hist, 0, sizeof(int) * e->S, s);
        if ((rc = launch_particles(e, true, s))) break;
        cudaEventRecord(a, s);
        for (int r = 0; r < reps && rc == BLOND_OK; ++r) rc = launch_particles(e, true, s);
        cudaEventRecord(b, s);
        if (rc) break;
        if (cudaEventSynchronize(b) != cudaSuccess) {
            rc = BLOND_ERR_CUDA;
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (ms / reps < best) {
            best = ms / reps;
            win = c;
            if (c.variant == 0) {
                win.threads = old.threads;
                win.bps = old.bps;
            }
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    // restore the state of the run
    cudaMemcpyAsync(e->dt, sdt, 8 * n, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(e->dE, sdE, esz * n, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(e->d_hist, shist, sizeof(int) * e->S, cudaMemcpyDeviceToDevice, s);
    const cudaError_t ce = cudaStreamSynchronize(s);
    free_ptr(sdt);
    free_ptr(sdE);
    free_ptr(shist);
    if (rc == BLOND_OK && ce != cudaSuccess) {
        set_error("engine_autotune: %s", cudaGetErrorString(ce));
        rc = BLOND_ERR_CUDA;
    }
    if (rc == BLOND_OK) rc = blond_engine_check(e, stream);
    const Cand& use = rc == BLOND_OK && best < 1e30 ? win : old;
    e->variant = use.variant;
    e->threads = use.threads;
    e->blocks_per_sm = use.bps;
    e->hist_mode = use.hist;
    e->ring = use.ring;
    e->cluster = use.cluster;
    e->graph_dirty = true;
    config[0] = use.variant;
    config[1] = use.variant == 0 ? kTmaThreads : use.threads;
    config[2] = use.variant == 0 ? 1 : use.bps;
    config[3] = use.hist;
    config[4] = use.ring;
    config[5] = use.cluster;
    config[6] = (int)cands.size();
    *best_ms = best < 1e30 ? best : 0.0;
    return rc;
}

// Capture (once per configuration) the graph of turns_per_graph turns and
// upload it to the device, so that the first replay costs no set-up time.
static int ensure_graph(blond_engine* e, cudaStream_t s) {
    const int K = e->turns_per_graph;
    if (!e->graph_dirty && e->graph_turns == K && e->graph) return BLOND_OK;
    int rc;
    // kernel attributes are set here, never inside the capture
    if ((rc = launch_particles(e, true, s, false))) return rc;
    if (e->has_fft && (rc = prepare_spectral())) return rc;
    if (e->graph) cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
    cudaGraph_t g;
    BB_CUDA(cudaStreamBeginCapture(e->cap_stream, cudaStreamCaptureModeThreadLocal));
    int lrc = BLOND_OK;
    for (int i = 0; i < K && lrc == BLOND_OK; ++i) lrc = launch_turn(e, e->cap_stream);
    cudaError_t ce = cudaStreamEndCapture(e->cap_stream, &g);
    if (lrc) return lrc;
    if (ce != cudaSuccess) {
        set_error("engine: graph capture failed: %s", cudaGetErrorString(ce));
        return BLOND_ERR_CUDA;
    }
    ce = cudaGraphInstantiate(&e->graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) {
        set_error("engine: graph instantiation failed: %s", cudaGetErrorString(ce));
        return BLOND_ERR_CUDA;
    }
    BB_CUDA(cudaGraphUpload(e->graph, s));
    e->graph_turns = K;
    e->graph_dirty = false;
    return BLOND_OK;
}

int blond_engine_prepare(blond_engine* e, void* stream) {
    BB_CHECK_ARG(e, "engine_prepare: null engine");
    int rc = check_ready(e);
    if (rc) return rc;
    if (e->turns_per_graph <= 1) return BLOND_OK;
    return ensure_graph(e, as_stream(stream));
}

int blond_engine_run(blond_engine* e, int64_t n_turns, void* stream) {
    BB_CHECK_ARG(e && n_turns >= 0, "engine_run: bad argument");
    int rc = check_ready(e);
    if (rc) return rc;
    BB_CHECK_SIZE(e->host_turn + n_turns <= e->n_turns,
                  "engine_run: turns %lld..%lld exceed the programme (%lld turns)",
                  (long long)e->host_turn, (long long)(e->host_turn + n_turns),
                  (long long)e->n_turns);
    if (n_turns == 0) return BLOND_OK;
    cudaStream_t s = as_stream(stream);
    const int K = e->turns_per_graph;
    int64_t done = 0;
    if (n_turns >= K && K > 1) {
        if ((rc = ensure_graph(e, s))) return rc;
        for (; done + K <= n_turns; done += K) BB_CUDA(cudaGraphLaunch(e->graph, s));
    }
    for (; done < n_turns; ++done) {
        rc = launch_turn(e, s);
        if (rc) return rc;
    }
    e->host_turn += n_turns;
    // the profile of the final coordinates (the histogram stays for the
    // next turn's head)
    return launch_profile(e, false, s);
}

// Turns on coordinates that live in host memory.  Every turn copies the
// beam in, runs the turn and copies it back, as a drop-in caller that keeps
// its arrays on the host sees it; the copies are pipelined in chunks over
// two copy streams (in and out directions concurrently) against the
// particle pass: chunk c is computed while c + 1 arrives and c - 1 leaves.
int blond_engine_track_host(blond_engine* e, double* host_dt, void* host_dE,
                            int64_t n_turns, int chunks, void* stream) {
    BB_CHECK_ARG(e && host_dt && host_dE && n_turns >= 0 && chunks >= 1 && chunks <= 256,
                 "engine_track_host: bad argument (chunks in 1..256)");
    int rc = check_ready(e);
    if (rc) return rc;
    BB_CHECK_SIZE(e->host_turn + n_turns <= e->n_turns,
                  "engine_track_host: turns exceed the programme");
    if (n_turns == 0) return BLOND_OK;
    cudaStream_t s = as_stream(stream);
    if (!e->io_in) {
        BB_CUDA(cudaStreamCreateWithFlags(&e->io_in, cudaStreamNonBlocking));
        BB_CUDA(cudaStreamCreateWithFlags(&e->io_out, cudaStreamNonBlocking));
    }
    while ((int)e->io_ev.size() < 3 * chunks + 1) {
        cudaEvent_t ev;
        BB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        e->io_ev.push_back(ev);
    }
    cudaEvent_t* ev_in = e->io_ev.data();
    cudaEvent_t* ev_done = ev_in + chunks;
    cudaEvent_t* ev_out = ev_done + chunks;
    cudaEvent_t ev_start = e->io_ev[3 * chunks];
    const int64_t n = e->n;
    const size_t esz = e->precision == BLOND_PREC_F64 ? sizeof(double) : sizeof(float);
    std::vector<int64_t> off((size_t)chunks + 1);
    for (int c = 0; c < chunks; ++c) off[c] = (n * c / chunks) & ~(int64_t)1;
    off[chunks] = n;
    double* ddt = static_cast<double*>(e->dt);
    char* ddE = static_cast<char*>(e->dE);
    char* hdE = static_cast<char*>(host_dE);
    // earlier work on the caller's stream touches the device coordinates
    BB_CUDA(cudaEventRecord(ev_start, s));
    BB_CUDA(cudaStreamWaitEvent(e->io_in, ev_start, 0));
    for (int64_t t = 0; t < n_turns; ++t) {
        for (int c = 0; c < chunks; ++c) {
            const int64_t o = off[c], m = off[c + 1] - off[c];
            // the previous turn's copy-out of this chunk has read it
            if (t > 0) BB_CUDA(cudaStreamWaitEvent(e->io_in, ev_out[c], 0));
            BB_CUDA(cudaMemcpyAsync(ddt + o, host_dt + o, sizeof(double) * m,
                                    cudaMemcpyHostToDevice, e->io_in));
            BB_CUDA(cudaMemcpyAsync(ddE + esz * o, hdE + esz * o, esz * m,
                                    cudaMemcpyHostToDevice, e->io_in));
            BB_CUDA(cudaEventRecord(ev_in[c], e->io_in));
        }
        if ((rc = launch_head(e, s))) return rc;
        for (int c = 0; c < chunks; ++c) {
            const int64_t o = off[c], m = off[c + 1] - off[c];
            BB_CUDA(cudaStreamWaitEvent(s, ev_in[c], 0));
            if (m > 0 && (rc = launch_particles_range(e, o, m, s))) return rc;
            BB_CUDA(cudaEventRecord(ev_done[c], s));
            BB_CUDA(cudaStreamWaitEvent(e->io_out, ev_done[c], 0));
            BB_CUDA(cudaMemcpyAsync(host_dt + o, ddt + o, sizeof(double) * m,
                                    cudaMemcpyDeviceToHost, e->io_out));
            BB_CUDA(cudaMemcpyAsync(hdE + esz * o, ddE + esz * o, esz * m,
                                    cudaMemcpyDeviceToHost, e->io_out));
            BB_CUDA(cudaEventRecord(ev_out[c], e->io_out));
        }
    }
    e->host_turn += n_turns;
    if ((rc = launch_profile(e, false, s))) return rc;
    // the caller's stream completes only after the last copy-out
    BB_CUDA(cudaStreamWaitEvent(s, ev_out[chunks - 1], 0));
    return BLOND_OK;
}

int blond_engine_time_kernels(blond_engine* e, int64_t n_turns, double* head_ms,
                              double* particles_ms, void* stream) {
    BB_CHECK_ARG(e && head_ms && particles_ms && n_turns >= 1,
                 "engine_time_kernels: bad argument");
    int rc = check_ready(e);
    if (rc) return rc;
    BB_CHECK_SIZE(e->host_turn + n_turns <= e->n_turns,
                  "engine_time_kernels: turns exceed the programme");
    cudaStream_t s = as_stream(stream);
    std::vector<cudaEvent_t> ev((size_t)(2 * n_turns + 1));
    for (auto& x : ev) BB_CUDA(cudaEventCreate(&x));
    rc = BLOND_OK;
    cudaEventRecord(ev[0], s);
    for (int64_t i = 0; i < n_turns && rc == BLOND_OK; ++i) {
        rc = launch_head(e, s);
        cudaEventRecord(ev[(size_t)(2 * i + 1)], s);
        if (rc == BLOND_OK) rc = launch_particles(e, true, s);
        cudaEventRecord(ev[(size_t)(2 * i + 2)], s);
    }
    cudaError_t ce = cudaEventSynchronize(ev.back());
    double h = 0, p = 0;
    for (int64_t i = 0; i < n_turns && ce == cudaSuccess; ++i) {
        float a = 0, b = 0;
        cudaEventElapsedTime(&a, ev[(size_t)(2 * i)], ev[(size_t)(2 * i + 1)]);
        cudaEventElapsedTime(&b, ev[(size_t)(2 * i + 1)], ev[(size_t)(2 * i + 2)]);
        h += a;
        p += b;
    }
    for (auto& x : ev) cudaEventDestroy(x);
    if (rc) return rc;
    if (ce != cudaSuccess) {
        set_error("engine_time_kernels: %s", cudaGetErrorString(ce));
        return BLOND_ERR_CUDA;
    }
    e->host_turn += n_turns;
    *head_ms = h;
    *particles_ms = p;
    return launch_profile(e, false, s);
}

int blond_engine_set_feedback(blond_engine* e, int machine, int delay, double gain,
                              double gain2, double alpha, int has_time_offset,
                              double time_offset, double bin_size, double ring_radius,
                              int sample_dE, const double* turn_table, const double* on_time,
                              int n_on_time, const double* state) {
    BB_CHECK_ARG(e, "engine_set_feedback: null engine");
    if (machine == 0) {
        e->has_fb = false;
        e->graph_dirty = true;
        return BLOND_OK;
    }
    BB_CHECK_ARG(machine >= BLOND_FB_LHC && machine <= BLOND_FB_PSB,
                 "engine_set_feedback: unknown machine %d", machine);
    BB_CHECK_ARG(turn_table && state, "engine_set_feedback: null table or state");
    BB_CHECK_ARG(e->rf_set, "engine_set_feedback: call set_rf first");
    BB_CHECK_ARG(sample_dE >= 1, "engine_set_feedback: sample_dE must be >= 1");
    BB_CHECK_ARG(machine != BLOND_FB_PSB || (on_time && n_on_time >= 1),
                 "engine_set_feedback: the PSB loop needs its on-time turns");
    const size_t cols = (size_t)FB_COLS + 2 * (size_t)e->n_rf;
    int rc;
    if ((rc = upload((void**)&e->d_fb_table, turn_table,
                     sizeof(double) * cols * (size_t)(e->n_turns + 1))))
        return rc;
    if ((rc = upload((void**)&e->d_fb_state, state,
                     sizeof(double) * ((size_t)FBS_DPHI_RF + e->n_rf))))
        return rc;
    if (machine == BLOND_FB_PSB &&
        (rc = upload((void**)&e->d_fb_on_time, on_time, sizeof(double) * n_on_time)))
        return rc;
    std::vector<double> zeros((size_t)(e->n_turns + 1) * 3, 0.0);
    if ((rc = upload((void**)&e->d_fb_trace, zeros.data(), sizeof(double) * zeros.size())))
        return rc;
    if (!e->d_fb_partials)
        BB_CUDA(cudaMalloc((void**)&e->d_fb_partials,
                           sizeof(double) * (kFbPartials + 2 * kFbMaxParts)));

    FeedbackArgs& a = e->fb;
    a = {};
    a.machine = machine;
    a.delay = delay;
    a.gain = gain;
    a.gain2 = gain2;
    a.alpha = alpha;
    a.has_time_offset = has_time_offset;
    a.time_offset = time_offset;
    a.bin_size = bin_size;
    a.ring_radius = ring_radius;
    a.sample_dE = sample_dE;
    a.n_on_time = machine == BLOND_FB_PSB ? n_on_time : 0;
    if (!e->d_fb_ticket) {
        BB_CUDA(cudaMalloc((void**)&e->d_fb_ticket, sizeof(int)));
        BB_CUDA(cudaMemset(e->d_fb_ticket, 0, sizeof(int)));
    }
    e->has_fb = true;
    e->graph_dirty = true;
    return BLOND_OK;
}

int blond_engine_get_feedback(blond_engine* e, double* state, double* omega_rf,
                              double* phi_rf, double* trace, void* stream) {
    BB_CHECK_ARG(e, "engine_get_feedback: null engine");
    BB_CHECK_ARG(e->has_fb, "engine_get_feedback: no beam-phase loop set");
    cudaStream_t s = as_stream(stream);
    const size_t cols = (size_t)(e->n_turns + 1) * e->n_rf;
    if (state)
        BB_CUDA(cudaMemcpyAsync(state, e->d_fb_state, sizeof(double) * (FBS_DPHI_RF + e->n_rf),
                                cudaMemcpyDeviceToDevice, s));
    if (omega_rf)
        BB_CUDA(cudaMemcpyAsync(omega_rf, e->d_om, sizeof(double) * cols,
                                cudaMemcpyDeviceToDevice, s));
    if (phi_rf)
        BB_CUDA(cudaMemcpyAsync(phi_rf, e->d_ph, sizeof(double) * cols,
                                cudaMemcpyDeviceToDevice, s));
    if (trace)
        BB_CUDA(cudaMemcpyAsync(trace, e->d_fb_trace, sizeof(double) * 3 * (e->n_turns + 1),
                                cudaMemcpyDeviceToDevice, s));
    return BLOND_OK;
}

int blond_engine_get_profile(blond_engine* e, double* out, void* stream) {
    BB_CHECK_ARG(e && out, "engine_get_profile: null pointer");
    BB_CUDA(cudaMemcpyAsync(out, e->d_profile, sizeof(double) * e->S,
                            cudaMemcpyDeviceToDevice, as_stream(stream)));
    return BLOND_OK;
}

int blond_engine_get_induced_voltage(blond_engine* e, double* out, void* stream) {
    BB_CHECK_ARG(e && out, "engine_get_induced_voltage: null pointer");
    BB_CUDA(cudaMemcpyAsync(out, e->d_vind, sizeof(double) * e->S,
                            cudaMemcpyDeviceToDevice, as_stream(stream)));
    return BLOND_OK;
}

int blond_engine_get_turn(blond_engine* e, int64_t* turn) {
    BB_CHECK_ARG(e && turn, "engine_get_turn: null pointer");
    *turn = e->host_turn;
    return BLOND_OK;
}

}  // extern "C"

// ===================================================== one turn, no allocation
// blond_turn_f64_noalloc runs the work of one fused turn (slice, induced
// voltage + table, particle pass, final profile) with every temporary held
// in a fixed file-scope device array instead of memory from cudaMalloc.
// It exists for callers that must not allocate device memory: a tracking
// step embedded in a host application that owns the device's memory (a
// control-room online model, a framework with its own pooling allocator)
// cannot call cudaMalloc, because the call can stall every stream on the
// device while it runs and it bypasses the host's memory accounting.
namespace bb {

// Largest profile the fixed scratch holds.
constexpr int kNoAllocMaxSlices = 16384;

struct NoAllocScratch {
    int hist[kNoAllocMaxSlices];              // integer slice counts
    double2 table[kNoAllocMaxSlices];         // interpolation table
    double bc[kNoAllocMaxSlices];             // bin centres (device copy)
    DriftTurn drift[2];                       // index 1 = this turn's drift
    double acc;                               // this turn's acceleration kick
    long long turn;                           // turn counter (0 -> 1)
    int err;                                  // bounded-wait error word
};

// ~448 KB per device that loads the library, held until the process exits.
// Shared by every call: calls that overlap on the GPU (e.g. on two
// streams) race on it.
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// Device address of the scratch on the current device, looked up once per
// device (cudaGetSymbolAddress; in host code the symbol's name is only a
// host-side stand-in, not a device address).
static NoAllocScratch* noalloc_scratch() {
    static NoAllocScratch* ptr[64] = {nullptr};
    static std::mutex mu;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        set_error("turn_noalloc: no current CUDA device");
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!ptr[dev]) {
        void* p = nullptr;
        const cudaError_t rc = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (rc != cudaSuccess || !p) {
            set_error("turn_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(rc));
            return nullptr;
        }
        ptr[dev] = reinterpret_cast<NoAllocScratch*>(p);
    }
    return ptr[dev];
}

}  // namespace bb

extern "C" int blond_turn_f64_noalloc(
    double* dt, double* dE, int64_t n, int n_rf, double charge, const double* voltage,
    const double* omega_rf, const double* phi_rf, double acc_kick, int solver,
    double t_rev, double length_ratio, double alpha_order, double eta_0, double eta_1,
    double eta_2, double alpha_0, double alpha_1, double alpha_2, double beta,
    double energy, double cut_left, double cut_right, int n_slices,
    const double* bin_centers, const double* impedance, int64_t n_fft, double iv_scale,
    double* profile_out, double* induced_voltage_out, void* stream) {
    using namespace bb;
    BB_CHECK_ARG(dt && dE && voltage && omega_rf && phi_rf && bin_centers && profile_out,
                 "turn_noalloc: null pointer");
    BB_CHECK_ARG(n >= 1, "turn_noalloc: n must be >= 1");
    BB_CHECK_ARG(solver >= 0 && solver <= 2, "turn_noalloc: solver %d", solver);
    BB_CHECK_ARG(aligned(dt, 16) && aligned(dE, 16),
                 "turn_noalloc: dt and dE must be 16-byte aligned");
    BB_CHECK_ARG(cut_right > cut_left, "turn_noalloc: cut_right <= cut_left");
    BB_CHECK_SIZE(n_rf >= 1 && n_rf <= kMaxRfEngine, "turn_noalloc: n_rf=%d not in [1, %d]",
                  n_rf, kMaxRfEngine);
    BB_CHECK_SIZE(n_slices >= 2 && n_slices <= kNoAllocMaxSlices,
                  "turn_noalloc: n_slices=%d exceeds the fixed scratch (2..%d slices); "
                  "use the engine API for longer profiles", n_slices, kNoAllocMaxSlices);
    SpecPlan plan = {};
    if (impedance) {
        BB_CHECK_ARG(induced_voltage_out, "turn_noalloc: null induced_voltage_out");
        if (!make_spec_plan(n_fft, plan)) {
            set_error("turn_noalloc: n_fft=%lld must be even, 5-smooth and <= %lld",
                      (long long)n_fft, (long long)kMaxClusterFFT);
            return BLOND_ERR_UNSUPPORTED;
        }
        BB_CHECK_SIZE(n_fft >= n_slices && plan.smem <= device_info().max_smem_optin,
                      "turn_noalloc: n_fft=%lld unsupported for %d slices",
                      (long long)n_fft, n_slices);
    }
    NoAllocScratch* sc = noalloc_scratch();
    if (!sc) return BLOND_ERR_CUDA;
    cudaStream_t s = as_stream(stream);

    // this turn's constants (drift.cpp:31-56 evaluated on the host, as the
    // engine does per turn), staged through pageable memory: the copy
    // returns once the bytes are staged, so the stack buffers may go
    struct Head {
        DriftTurn drift[2];
        double acc;
        long long turn;
        int err;
    } h = {};
    DriftTurn& d = h.drift[1];
    d.Tr = t_rev * length_ratio;
    d.simple = d.Tr * eta_0 / (beta * beta * energy);
    const double coeff = 1. / (beta * beta * energy);
    d.e0 = eta_0 * coeff;
    d.e1 = eta_1 * coeff * coeff;
    d.e2 = eta_2 * coeff * coeff * coeff;
    d.ib2 = 1 / (beta * beta);
    d.ie2 = 1 / (energy * energy);
    d.energy = energy;
    d.a0 = alpha_0;
    d.a1 = alpha_1;
    d.a2 = alpha_2;
    h.drift[0] = d;
    h.acc = acc_kick;
    h.turn = 0;
    h.err = 0;
    static_assert(offsetof(NoAllocScratch, acc) ==
                      offsetof(NoAllocScratch, drift) + 2 * sizeof(DriftTurn),
                  "scratch header layout");
    BB_CUDA(cudaMemcpyAsync(&sc->drift[0], &h.drift[0], sizeof(h.drift), cudaMemcpyHostToDevice, s));
    BB_CUDA(cudaMemcpyAsync(&sc->acc, &h.acc, sizeof(double), cudaMemcpyHostToDevice, s));
    BB_CUDA(cudaMemcpyAsync(&sc->turn, &h.turn, sizeof(long long), cudaMemcpyHostToDevice, s));
    BB_CUDA(cudaMemcpyAsync(&sc->err, &h.err, sizeof(int), cudaMemcpyHostToDevice, s));
    BB_CUDA(cudaMemcpyAsync(sc->bc, bin_centers, sizeof(double) * n_slices,
                            cudaMemcpyHostToDevice, s));
    // the histogram must start at zero; the previous call leaves its last
    // turn's counts behind
    BB_CUDA(cudaMemsetAsync(sc->hist, 0, sizeof(int) * n_slices, s));

    // an engine description on the stack pointing at the caller's buffers
    // and the fixed scratch (no allocation: none of the set-up calls run)
    blond_engine e;
    e.precision = BLOND_PREC_F64;
    e.n_rf = n_rf;
    e.solver = solver;
    e.S = n_slices;
    cudaGetDevice(&e.device);
    e.n_turns = 1;
    e.charge = charge;
    e.d_V = const_cast<double*>(voltage);
    e.d_om = const_cast<double*>(omega_rf);
    e.d_ph = const_cast<double*>(phi_rf);
    e.d_acc = &sc->acc;
    e.d_drift = sc->drift;
    e.order = alpha_order == 0 ? 0 : (alpha_order == 1 ? 1 : 2);
    e.rf_set = e.drift_set = e.slicing_set = true;
    e.cut_left = cut_left;
    e.cut_right = cut_right;
    e.inv_w = n_slices / (cut_right - cut_left);
    e.d_bc = sc->bc;
    e.bc0 = bin_centers[0];
    e.lik_inv_w = (n_slices - 1) / (bin_centers[n_slices - 1] - bin_centers[0]);
    e.bw = 1.0 / e.lik_inv_w;
    e.dbc = bin_centers[1] - bin_centers[0];
    e.has_fft = impedance != nullptr;
    e.plan = plan;
    e.d_H = reinterpret_cast<double2*>(const_cast<double*>(impedance));
    e.iv_scale = iv_scale;
    e.d_turn = &sc->turn;
    e.d_err = &sc->err;
    e.d_hist = sc->hist;
    e.d_profile = profile_out;
    e.d_vind = induced_voltage_out;
    e.d_table = sc->table;
    e.dt = dt;
    e.dE = dE;
    e.n = n;
    e.variant = 1;  // plain-load particle pass, the engine's FP64 choice

    int rc;
    if ((rc = launch_particles(&e, false, s))) return rc;  // slice the input
    if ((rc = launch_head(&e, s))) return rc;              // profile, V, table
    if ((rc = launch_particles(&e, true, s))) return rc;   // the turn
    return launch_profile(&e, false, s);                   // final profile
}

// ============================================================ batched beams
// Many independent beams (ragged particle counts, own RF programme, slicing
// window and impedance each) tracked together: ONE particle launch and ONE
// head launch per turn for the whole batch.  Particles are concatenated;
// a chunk table cuts every beam into pieces of at most kBatchChunk
// particles, each piece processed by one block with its beam's constants in
// shared memory and a private shared-memory histogram flushed to the beam's
// global histogram.  The head kernel runs one cluster per beam.  Each beam
// follows exactly the arithmetic of the single-beam engine (track_pair).
namespace bb {

constexpr int kBatchChunk = 32768;
constexpr int kBatchThreads = 512;

struct BatchArgs {
    void* dt;
    void* dE;
    const long long* chunk_start;
    const int* chunk_beam;
    const int* chunk_count;
    int n_chunks;
    int n_rf;
    double charge;
    const double* V;  // [B][n_turns+1][n_rf]
    const double* om;
    const double* ph;
    const double* acc;          // [B][n_turns]
    const DriftTurn* drift;     // [B][n_turns+1]
    int64_t n_turns;
    int order;
    const long long* turn;
    int S;
    const double* cut_left;     // [B]
    const double* inv_w;        // [B]
    const double* bc0;          // [B]
    const double* lik_inv_w;    // [B]
    const double* bw;           // [B]
    int* hist;                  // [B][S]
    const void* table;          // [B][S]
};

template <int PREC, int SOLVER, bool LIK, bool KICK>
__global__ void __launch_bounds__(kBatchThreads, 2)
particle_kernel_batch(const BatchArgs a) {
    using E = typename Coord<PREC>::E;
    extern __shared__ int sh[];
    __shared__ TurnConsts c;
    long long t = a.turn ? (*a.turn - 1) : 0;
    if (t < 0) t = 0;
    if (t >= a.n_turns) t = a.n_turns - 1;
    double* dt = reinterpret_cast<double*>(a.dt);
    E* dE = reinterpret_cast<E*>(a.dE);
    const int S = a.S;
    const uint64_t pol = evict_first_policy();
    for (int ch = blockIdx.x; ch < a.n_chunks; ch += gridDim.x) {
        const int b = a.chunk_beam[ch];
        const long long start = a.chunk_start[ch];
        const int count = a.chunk_count[ch];
        if (KICK) {
            const long long rb = (long long)b * (a.n_turns + 1);
            for (int j = threadIdx.x; j < a.n_rf; j += blockDim.x) {
                c.V[j] = a.V[(rb + t) * a.n_rf + j];
                c.Vf[j] = (float)c.V[j];
                c.om[j] = a.om[(rb + t) * a.n_rf + j];
                c.ph[j] = a.ph[(rb + t) * a.n_rf + j];
            }
            if (threadIdx.x == 0) {
                c.acc = a.acc[(long long)b * a.n_turns + t];
                c.d = a.drift[rb + t + 1];
            }
        }
        for (int k = threadIdx.x; k < S; k += blockDim.x) sh[k] = 0;
        __syncthreads();
        ParticleArgs pa = {};
        pa.n_rf = a.n_rf;
        pa.charge = a.charge;
        pa.S = S;
        pa.bc0 = a.bc0[b];
        pa.lik_inv_w = a.lik_inv_w[b];
        pa.bw = a.bw[b];
        pa.table = LIK ? static_cast<const char*>(a.table) +
                             (long long)b * S * (PREC == PREC_F64 ? 16 : 8)
                       : nullptr;
        const double cl = a.cut_left[b], iw = a.inv_w[b];
        // four particles per thread and iteration (i + q * blockDim, q < 4),
        // all loads issued before any arithmetic: with two, each SM had
        // only ~16 KB of loads in flight, which caps HBM near 2.4 TB/s
        const int bd = blockDim.x;
        for (int i = threadIdx.x; i < count; i += 4 * bd) {
            // F32P64: thread 0 prefetches the block's next iteration into L2
            // (C3: 2.059 -> 2.040 ms per turn)
            if (PREC == PREC_F32P64 && threadIdx.x == 0 && i + 4 * bd < count) {
                const long long lo = start + i + 4LL * bd;
                const long long hi = start + min((long long)count, (long long)i + 8LL * bd);
                l2_prefetch_range(dt + lo, dt + hi, pol);
                l2_prefetch_range(dE + lo, dE + hi, pol);
            }
            double t[4];
            E e[4];
            bool in[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                in[q] = i + q * bd < count;
                const long long g = start + i + (in[q] ? q * bd : 0);
                t[q] = stream_load(dt + g, pol);
                e[q] = stream_load(dE + g, pol);
            }
            if (KICK) {
                track_pair<PREC, SOLVER, LIK>(t[0], t[1], e[0], e[1], c, pa, a.order);
                track_pair<PREC, SOLVER, LIK>(t[2], t[3], e[2], e[3], c, pa, a.order);
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if (in[q]) {
                        stream_store(dt + start + i + q * bd, t[q], pol);
                        stream_store(dE + start + i + q * bd, e[q], pol);
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int bq = in[q] ? engine_bin(t[q], cl, iw, S) : -1;
                if (bq >= 0) atomicAdd(&sh[bq], 1);
            }
        }
        __syncthreads();
        for (int k = threadIdx.x; k < S; k += blockDim.x) {
            const int v = sh[k];
            if (v) atomicAdd(&a.hist[(long long)b * S + k], v);
        }
        __syncthreads();  // shared histogram and constants are reused
    }
}

}  // namespace bb

struct blond_batch {
    int precision = 0, B = 0, n_rf = 0, solver = 0, S = 0, device = 0;
    int64_t n_turns = 0;
    double charge = 1.0;
    int order = 0;
    double* d_V = nullptr;
    double* d_om = nullptr;
    double* d_ph = nullptr;
    double* d_acc = nullptr;
    bb::DriftTurn* d_drift = nullptr;
    long long* d_chunk_start = nullptr;
    int* d_chunk_beam = nullptr;
    int* d_chunk_count = nullptr;
    int n_chunks = 0;
    double* d_cl = nullptr;
    double* d_inv_w = nullptr;
    double* d_bc0 = nullptr;
    double* d_lik_inv_w = nullptr;
    double* d_bw = nullptr;
    double* d_bc = nullptr;
    bool has_fft = false;
    bb::SpecPlan plan = {};
    double2* d_H = nullptr;
    double* d_scale = nullptr;
    double2* d_tw = nullptr;
    int* d_hist = nullptr;
    double* d_profile = nullptr;
    double* d_vind = nullptr;
    void* d_table = nullptr;
    long long* d_turn = nullptr;
    long long host_turn = 0;
    void* dt = nullptr;
    void* dE = nullptr;
    int64_t n_total = 0;
    bool rf_set = false, drift_set = false, slicing_set = false;
    int turns_per_graph = 50;
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_turns = 0;
    bool graph_dirty = true;
};

namespace bb {

static BatchArgs batch_args(blond_batch* q) {
    BatchArgs a = {};
    a.dt = q->dt;
    a.dE = q->dE;
    a.chunk_start = q->d_chunk_start;
    a.chunk_beam = q->d_chunk_beam;
    a.chunk_count = q->d_chunk_count;
    a.n_chunks = q->n_chunks;
    a.n_rf = q->n_rf;
    a.charge = q->charge;
    a.V = q->d_V;
    a.om = q->d_om;
    a.ph = q->d_ph;
    a.acc = q->d_acc;
    a.drift = q->d_drift;
    a.n_turns = q->n_turns;
    a.order = q->order;
    a.turn = q->d_turn;
    a.S = q->S;
    a.cut_left = q->d_cl;
    a.inv_w = q->d_inv_w;
    a.bc0 = q->d_bc0;
    a.lik_inv_w = q->d_lik_inv_w;
    a.bw = q->d_bw;
    a.hist = q->d_hist;
    a.table = q->d_table;
    return a;
}

template <int PREC, int SOLVER, bool LIK, bool KICK>
static int launch_batch_t(blond_batch* q, cudaStream_t s, bool launch) {
    static bool done[64] = {false};
    auto k = particle_kernel_batch<PREC, SOLVER, LIK, KICK>;
    int rc;
    if ((rc = allow_max_smem(k, done))) return rc;
    if (!launch) return BLOND_OK;
    const int smem = (int)sizeof(int) * q->S;
    const int grid = std::max(1, std::min(q->n_chunks, device_info().sm_count * 2));
    k<<<grid, kBatchThreads, smem, s>>>(batch_args(q));
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

template <int PREC>
static int launch_batch_p(blond_batch* q, bool kick, cudaStream_t s, bool launch) {
    if (!kick) return launch_batch_t<PREC, 0, false, false>(q, s, launch);
    const bool lik = q->has_fft;
    switch (q->solver) {
        case 0:
            return lik ? launch_batch_t<PREC, 0, true, true>(q, s, launch)
                       : launch_batch_t<PREC, 0, false, true>(q, s, launch);
        case 1:
            return lik ? launch_batch_t<PREC, 1, true, true>(q, s, launch)
                       : launch_batch_t<PREC, 1, false, true>(q, s, launch);
        default:
            return lik ? launch_batch_t<PREC, 2, true, true>(q, s, launch)
                       : launch_batch_t<PREC, 2, false, true>(q, s, launch);
    }
}

static int launch_batch(blond_batch* q, bool kick, cudaStream_t s, bool launch = true) {
    if (q->precision == BLOND_PREC_F64) return launch_batch_p<PREC_F64>(q, kick, s, launch);
    return launch_batch_p<PREC_F32P64>(q, kick, s, launch);
}

static int launch_batch_profile(blond_batch* q, bool clear, cudaStream_t s) {
    const int total = q->B * q->S;
    const int threads = 256;
    const int grid = std::min(1024, (total + threads - 1) / threads);
    profile_kernel<<<grid, threads, 0, s>>>(q->d_hist, q->d_profile, total, clear ? 1 : 0,
                                            clear ? q->d_turn : nullptr);
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

static int launch_batch_head(blond_batch* q, cudaStream_t s) {
    if (!q->has_fft) return launch_batch_profile(q, true, s);
    SpecParams P = {};
    P.p = q->plan;
    P.mode = SPEC_FORWARD | SPEC_MULTIPLY | SPEC_INVERSE;
    P.in_i32 = q->d_hist;
    P.n_in = q->S;
    P.profile_out = q->d_profile;
    P.H = q->d_H;
    P.out = q->d_vind;
    P.n_out = q->S;
    P.table = q->d_table;
    P.table_f32 = q->precision == BLOND_PREC_F32P64;
    P.charge = q->charge;
    P.bc = q->d_bc;
    P.turn = q->d_turn;
    P.bump_turn = 1;
    P.twg = q->d_tw;
    P.batch = q->B;
    P.beam_scale = q->d_scale;
    P.beam_inv_w = q->d_lik_inv_w;
    return launch_spectral(P, s);
}

static int batch_ready(blond_batch* q) {
    if (!q->rf_set || !q->drift_set || !q->slicing_set || !q->dt) {
        set_error("batch: set_rf, set_drift, set_slicing and bind_beams must all be called "
                  "before tracking");
        return BLOND_ERR_STATE;
    }
    return BLOND_OK;
}

static int batch_turn(blond_batch* q, cudaStream_t s) {
    int rc = launch_batch_head(q, s);
    if (rc) return rc;
    return launch_batch(q, true, s);
}

}  // namespace bb

extern "C" {

int blond_batch_create(blond_batch** out, int precision, int n_beams, int n_rf, int solver,
                       int n_slices) {
    using namespace bb;
    BB_CHECK_ARG(out, "batch_create: null output");
    BB_CHECK_ARG(precision == BLOND_PREC_F64 || precision == BLOND_PREC_F32P64,
                 "batch_create: unknown precision %d", precision);
    BB_CHECK_SIZE(n_beams >= 1, "batch_create: n_beams must be >= 1");
    BB_CHECK_SIZE(n_rf >= 1 && n_rf <= kMaxRfEngine, "batch_create: n_rf=%d", n_rf);
    BB_CHECK_ARG(solver >= 0 && solver <= 2, "batch_create: solver %d", solver);
    const int max_s = (device_info().max_smem_optin - (int)sizeof(TurnConsts) - 1024) / 8;
    BB_CHECK_SIZE(n_slices >= 2 && n_slices <= max_s, "batch_create: n_slices=%d not in [2, %d]",
                  n_slices, max_s);
    blond_batch* q = new blond_batch();
    q->precision = precision;
    q->B = n_beams;
    q->n_rf = n_rf;
    q->solver = solver;
    q->S = n_slices;
    cudaGetDevice(&q->device);
    const size_t bs = (size_t)n_beams * n_slices;
    int rc = BLOND_OK;
    if (cudaMalloc(&q->d_turn, sizeof(long long)) != cudaSuccess ||
        cudaMalloc(&q->d_hist, sizeof(int) * bs) != cudaSuccess ||
        cudaMalloc(&q->d_profile, sizeof(double) * bs) != cudaSuccess ||
        cudaMalloc(&q->d_vind, sizeof(double) * bs) != cudaSuccess ||
        cudaMalloc(&q->d_table, sizeof(double2) * bs) != cudaSuccess ||
        cudaStreamCreateWithFlags(&q->cap_stream, cudaStreamNonBlocking) != cudaSuccess) {
        set_error("batch_create: allocation failed");
        rc = BLOND_ERR_CUDA;
    } else {
        cudaMemset(q->d_turn, 0, sizeof(long long));
        cudaMemset(q->d_hist, 0, sizeof(int) * bs);
        cudaMemset(q->d_profile, 0, sizeof(double) * bs);
        cudaMemset(q->d_vind, 0, sizeof(double) * bs);
        cudaMemset(q->d_table, 0, sizeof(double2) * bs);
        if (cudaDeviceSynchronize() != cudaSuccess) {
            set_error("batch_create: device error");
            rc = BLOND_ERR_CUDA;
        }
    }
    if (rc) {
        blond_batch_destroy(q);
        return rc;
    }
    *out = q;
    return BLOND_OK;
}

int blond_batch_destroy(blond_batch* q) {
    using namespace bb;
    if (!q) return BLOND_OK;
    if (q->graph) cudaGraphExecDestroy(q->graph);
    if (q->cap_stream) cudaStreamDestroy(q->cap_stream);
    for (void* p : {(void*)q->d_V, (void*)q->d_om, (void*)q->d_ph, (void*)q->d_acc,
                    (void*)q->d_drift, (void*)q->d_chunk_start, (void*)q->d_chunk_beam,
                    (void*)q->d_chunk_count, (void*)q->d_cl, (void*)q->d_inv_w,
                    (void*)q->d_bc0, (void*)q->d_lik_inv_w, (void*)q->d_bw, (void*)q->d_bc,
                    (void*)q->d_H, (void*)q->d_scale, (void*)q->d_tw, (void*)q->d_hist,
                    (void*)q->d_profile, (void*)q->d_vind, q->d_table, (void*)q->d_turn})
        free_ptr(p);
    delete q;
    return BLOND_OK;
}

int blond_batch_set_rf(blond_batch* q, int64_t n_turns, const double* V, const double* om,
                       const double* ph, const double* acc, double charge) {
    using namespace bb;
    BB_CHECK_ARG(q && V && om && ph && acc && n_turns >= 1, "batch_set_rf: bad argument");
    const size_t cols = (size_t)q->B * (n_turns + 1) * q->n_rf;
    int rc;
    if ((rc = upload((void**)&q->d_V, V, sizeof(double) * cols))) return rc;
    if ((rc = upload((void**)&q->d_om, om, sizeof(double) * cols))) return rc;
    if ((rc = upload((void**)&q->d_ph, ph, sizeof(double) * cols))) return rc;
    if ((rc = upload((void**)&q->d_acc, acc, sizeof(double) * q->B * n_turns))) return rc;
    q->n_turns = n_turns;
    q->charge = charge;
    q->rf_set = true;
    q->graph_dirty = true;
    return BLOND_OK;
}

int blond_batch_set_drift(blond_batch* q, double length_ratio, double alpha_order,
                          const double* t_rev, const double* eta_0, const double* eta_1,
                          const double* eta_2, const double* alpha_0, const double* alpha_1,
                          const double* alpha_2, const double* beta, const double* energy) {
    using namespace bb;
    BB_CHECK_ARG(q && t_rev && eta_0 && eta_1 && eta_2 && alpha_0 && alpha_1 && alpha_2 &&
                     beta && energy && q->rf_set,
                 "batch_set_drift: bad argument (set_rf first)");
    const size_t nt = (size_t)q->n_turns + 1, total = nt * q->B;
    std::vector<DriftTurn> h(total);
    for (size_t i = 0; i < total; ++i) {
        // drift.cpp:31-56, as blond_engine_set_drift
        DriftTurn d = {};
        d.Tr = t_rev[i] * length_ratio;
        d.simple = d.Tr * eta_0[i] / (beta[i] * beta[i] * energy[i]);
        const double coeff = 1. / (beta[i] * beta[i] * energy[i]);
        d.e0 = eta_0[i] * coeff;
        d.e1 = eta_1[i] * coeff * coeff;
        d.e2 = eta_2[i] * coeff * coeff * coeff;
        d.ib2 = 1 / (beta[i] * beta[i]);
        d.ie2 = 1 / (energy[i] * energy[i]);
        d.energy = energy[i];
        d.a0 = alpha_0[i];
        d.a1 = alpha_1[i];
        d.a2 = alpha_2[i];
        h[i] = d;
    }
    q->order = alpha_order == 0 ? 0 : (alpha_order == 1 ? 1 : 2);
    int rc = upload((void**)&q->d_drift, h.data(), sizeof(DriftTurn) * total);
    if (rc) return rc;
    q->drift_set = true;
    q->graph_dirty = true;
    return BLOND_OK;
}

int blond_batch_set_slicing(blond_batch* q, const double* cut_left, const double* cut_right,
                            const double* bc) {
    using namespace bb;
    BB_CHECK_ARG(q && cut_left && cut_right && bc, "batch_set_slicing: null pointer");
    const int B = q->B, S = q->S;
    std::vector<double> cl(B), iw(B), b0(B), liw(B), bw(B);
    for (int b = 0; b < B; ++b) {
        BB_CHECK_ARG(cut_right[b] > cut_left[b], "batch_set_slicing: beam %d cut_right <= "
                     "cut_left", b);
        const double* c = bc + (size_t)b * S;
        cl[b] = cut_left[b];
        iw[b] = S / (cut_right[b] - cut_left[b]);             // histogram.cpp:30
        b0[b] = c[0];
        liw[b] = (S - 1) / (c[S - 1] - c[0]);                 // linear_interp_kick.cpp:31-33
        bw[b] = 1.0 / liw[b];
    }
    int rc;
    if ((rc = upload((void**)&q->d_cl, cl.data(), sizeof(double) * B))) return rc;
    if ((rc = upload((void**)&q->d_inv_w, iw.data(), sizeof(double) * B))) return rc;
    if ((rc = upload((void**)&q->d_bc0, b0.data(), sizeof(double) * B))) return rc;
    if ((rc = upload((void**)&q->d_lik_inv_w, liw.data(), sizeof(double) * B))) return rc;
    if ((rc = upload((void**)&q->d_bw, bw.data(), sizeof(double) * B))) return rc;
    if ((rc = upload((void**)&q->d_bc, bc, sizeof(double) * (size_t)B * S))) return rc;
    q->slicing_set = true;
    q->graph_dirty = true;
    return BLOND_OK;
}

int blond_batch_set_impedance(blond_batch* q, int64_t n_fft, const double* Z,
                              const double* scale) {
    using namespace bb;
    BB_CHECK_ARG(q && Z && scale, "batch_set_impedance: null pointer");
    SpecPlan plan;
    if (!make_spec_plan(n_fft, plan)) {
        set_error("batch_set_impedance: n_fft=%lld must be even, 5-smooth and <= %lld",
                  (long long)n_fft, (long long)kMaxClusterFFT);
        return BLOND_ERR_UNSUPPORTED;
    }
    BB_CHECK_SIZE(n_fft >= q->S && plan.smem <= device_info().max_smem_optin,
                  "batch_set_impedance: n_fft=%lld unsupported for %d slices",
                  (long long)n_fft, q->S);
    std::vector<double> sc(q->B);
    for (int b = 0; b < q->B; ++b) sc[b] = -scale[b] / (double)plan.M;
    int rc;
    if ((rc = upload((void**)&q->d_H, Z, sizeof(double2) * (size_t)q->B * (n_fft / 2 + 1))))
        return rc;
    if ((rc = upload((void**)&q->d_scale, sc.data(), sizeof(double) * q->B))) return rc;
    free_ptr(q->d_tw);
    q->d_tw = nullptr;
    if ((rc = make_spec_twiddles(plan, &q->d_tw))) return rc;
    q->plan = plan;
    q->has_fft = true;
    q->graph_dirty = true;
    return BLOND_OK;
}

int blond_batch_bind_beams(blond_batch* q, void* dt, void* dE, const int64_t* offsets) {
    using namespace bb;
    BB_CHECK_ARG(q && dt && dE && offsets, "batch_bind_beams: null pointer");
    BB_CHECK_ARG(aligned(dt, 8) && aligned(dE, 8), "batch_bind_beams: misaligned arrays");
    std::vector<long long> cs;
    std::vector<int> cb, cc;
    for (int b = 0; b < q->B; ++b) {
        BB_CHECK_ARG(offsets[b + 1] >= offsets[b], "batch_bind_beams: offsets decrease");
        for (int64_t s0 = offsets[b]; s0 < offsets[b + 1]; s0 += kBatchChunk) {
            cs.push_back(s0);
            cb.push_back(b);
            cc.push_back((int)std::min<int64_t>(kBatchChunk, offsets[b + 1] - s0));
        }
    }
    int rc;
    q->n_chunks = (int)cs.size();
    if (q->n_chunks) {
        if ((rc = upload((void**)&q->d_chunk_start, cs.data(), sizeof(long long) * cs.size())))
            return rc;
        if ((rc = upload((void**)&q->d_chunk_beam, cb.data(), sizeof(int) * cb.size()))) return rc;
        if ((rc = upload((void**)&q->d_chunk_count, cc.data(), sizeof(int) * cc.size())))
            return rc;
    }
    q->dt = dt;
    q->dE = dE;
    q->n_total = offsets[q->B];
    q->graph_dirty = true;
    return BLOND_OK;
}

int blond_batch_set_turn(blond_batch* q, int64_t turn, void* stream) {
    using namespace bb;
    BB_CHECK_ARG(q && turn >= 0, "batch_set_turn: bad argument");
    const long long t = turn;
    BB_CUDA(cudaMemcpyAsync(q->d_turn, &t, sizeof(t), cudaMemcpyHostToDevice,
                            as_stream(stream)));
    BB_CUDA(cudaStreamSynchronize(as_stream(stream)));
    q->host_turn = turn;
    return BLOND_OK;
}

int blond_batch_slice(blond_batch* q, void* stream) {
    using namespace bb;
    BB_CHECK_ARG(q, "batch_slice: null batch");
    int rc = batch_ready(q);
    if (rc) return rc;
    cudaStream_t s = as_stream(stream);
    BB_CUDA(cudaMemsetAsync(q->d_hist, 0, sizeof(int) * (size_t)q->B * q->S, s));
    if ((rc = launch_batch(q, false, s))) return rc;
    return launch_batch_profile(q, false, s);
}

int blond_batch_prepare(blond_batch* q, void* stream) {
    using namespace bb;
    BB_CHECK_ARG(q, "batch_prepare: null batch");
    int rc = batch_ready(q);
    if (rc) return rc;
    const int K = q->turns_per_graph;
    if (K <= 1 || (!q->graph_dirty && q->graph)) return BLOND_OK;
    cudaStream_t s = as_stream(stream);
    // kernel attributes are set here, never inside the capture
    if ((rc = launch_batch(q, true, s, false))) return rc;
    if (q->has_fft && (rc = prepare_spectral())) return rc;
    if (q->graph) cudaGraphExecDestroy(q->graph);
    q->graph = nullptr;
    cudaGraph_t g;
    BB_CUDA(cudaStreamBeginCapture(q->cap_stream, cudaStreamCaptureModeThreadLocal));
    int lrc = BLOND_OK;
    for (int i = 0; i < K && lrc == BLOND_OK; ++i) lrc = batch_turn(q, q->cap_stream);
    cudaError_t ce = cudaStreamEndCapture(q->cap_stream, &g);
    if (lrc) return lrc;
    if (ce != cudaSuccess) {
        set_error("batch: graph capture failed: %s", cudaGetErrorString(ce));
        return BLOND_ERR_CUDA;
    }
    ce = cudaGraphInstantiate(&q->graph, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) {
        set_error("batch: graph instantiation failed: %s", cudaGetErrorString(ce));
        return BLOND_ERR_CUDA;
    }
    BB_CUDA(cudaGraphUpload(q->graph, s));
    q->graph_turns = K;
    q->graph_dirty = false;
    return BLOND_OK;
}

int blond_batch_run(blond_batch* q, int64_t n_turns, void* stream) {
    using namespace bb;
    BB_CHECK_ARG(q && n_turns >= 0, "batch_run: bad argument");
    int rc = batch_ready(q);
    if (rc) return rc;
    BB_CHECK_SIZE(q->host_turn + n_turns <= q->n_turns,
                  "batch_run: turns exceed the programme (%lld turns)", (long long)q->n_turns);
    if (n_turns == 0) return BLOND_OK;
    cudaStream_t s = as_stream(stream);
    const int K = q->turns_per_graph;
    int64_t done = 0;
    if (n_turns >= K && K > 1) {
        if ((rc = blond_batch_prepare(q, stream))) return rc;
        for (; done + K <= n_turns; done += K) BB_CUDA(cudaGraphLaunch(q->graph, s));
    }
    for (; done < n_turns; ++done)
        if ((rc = batch_turn(q, s))) return rc;
    q->host_turn += n_turns;
    return launch_batch_profile(q, false, s);
}

int blond_batch_tune(blond_batch* q, int turns_per_graph) {
    BB_CHECK_ARG(q && turns_per_graph >= 0, "batch_tune: bad argument");
    if (turns_per_graph) q->turns_per_graph = turns_per_graph;
    q->graph_dirty = true;
    return BLOND_OK;
}

int blond_batch_get_profiles(blond_batch* q, double* out, void* stream) {
    using namespace bb;
    BB_CHECK_ARG(q && out, "batch_get_profiles: null pointer");
    BB_CUDA(cudaMemcpyAsync(out, q->d_profile, sizeof(double) * (size_t)q->B * q->S,
                            cudaMemcpyDeviceToDevice, as_stream(stream)));
    return BLOND_OK;
}

int blond_batch_get_induced_voltages(blond_batch* q, double* out, void* stream) {
    using namespace bb;
    BB_CHECK_ARG(q && out, "batch_get_induced_voltages: null pointer");
    BB_CUDA(cudaMemcpyAsync(out, q->d_vind, sizeof(double) * (size_t)q->B * q->S,
                            cudaMemcpyDeviceToDevice, as_stream(stream)));
    return BLOND_OK;
}

}  // extern "C"
