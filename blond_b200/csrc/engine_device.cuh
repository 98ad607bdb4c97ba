// Device side of the fused turn engine, shared by the single-beam engine
// (engine.cu) and the batched engine (batch.cu): per-turn constants, the
// per-particle turn (induced kick, RF kick, drift) in every precision mode,
// the slice deposit layouts, the streaming load/store helpers and the
// particle-pass kernels, plus the host helpers both engines use.
#pragma once

#include "spectral.cuh"
#include "feedback.cuh"

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <mutex>
#include <set>
#include <type_traits>
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
    // Q32P64: the energy unit (eV per count of the int32 dE) and its inverse
    double lsb, inv_lsb;
    // sticky error word: bit 0 a bounded wait gave up, bit 1 an energy left
    // its 32-bit grid (Q32P64)
    int* err;
    // interpolated tracker: the RF kick and the acceleration kick are part
    // of the interpolation table, so the pass runs with n_rf = 0 and acc 0
    int interp;
    // smooth slicing: a separate deposit pass makes the profile, this pass
    // deposits nothing
    int no_deposit;
    // shared-table pass (particle_kernel_stab): the induced voltage the head
    // wrote, and the slicing frame whose numpy.linspace midpoints are the
    // bin centres (bc_step = (cut_right - cut_left) / S)
    const double* vind;
    double cut_right, bc_step;
    // shared-table pass: thread 0 also prefetches the block's slice one
    // iteration beyond the ring into L2
    int l2_ahead;
};

enum { PREC_F64 = 0, PREC_F32P64 = 1, PREC_Q32P64 = 2 };

template <int PREC>
struct Coord;
template <> struct Coord<PREC_F64> { using E = double; };
template <> struct Coord<PREC_F32P64> { using E = float; };
template <> struct Coord<PREC_Q32P64> { using E = int; };

// Interpolation-table entry of the induced kick: {slope, offset} in float64
// (linear_interp_kick.cpp:41-47) for F64 and Q32P64, {qV_k, slope_k} in
// float32 for F32P64.
template <int PREC> struct TableEntry { using T = double2; };
template <> struct TableEntry<PREC_F32P64> { using T = float2; };

enum { ERR_WAIT = 1, ERR_ENERGY_RANGE = 2 };

// Q32P64: the energy in eV of a count on the grid.
template <int PREC>
__device__ __forceinline__ double energy_value(typename Coord<PREC>::E e, const ParticleArgs& a) {
    if constexpr (PREC == PREC_Q32P64) return __dmul_rn((double)e, a.lsb);
    else return (double)e;
}

// Q32P64: counts + this turn's float64 energy increment, rounded once to
// the grid.  A result beyond +-(2^31 - 1) counts (or a NaN increment) sets
// the error word and saturates.
__device__ __forceinline__ int q32_add(int q, double inc, const ParticleArgs& a) {
    long long r = (long long)q + __double2ll_rn(__dmul_rn(inc, a.inv_lsb));
    if (r > 2147483647LL || r < -2147483647LL) {
        if (a.err) atomicOr(a.err, ERR_ENERGY_RANGE);
        r = r > 0 ? 2147483647LL : -2147483647LL;
    }
    return (int)r;
}

// Table sources of the induced kick: the global table the head wrote, or a
// copy in shared memory (F64 / Q32P64: the induced voltage only, entries
// formed per particle with lik_entry; F32P64: the float2 table itself).
// TAB_ENTRIES: the table's own entries in shared memory (the batched pass
// copies its beam's short table per chunk).
enum { TAB_GLOBAL = 0, TAB_SHARED = 1, TAB_ENTRIES = 2 };

// numpy.linspace midpoint k (linspace_centre) with the step precomputed.
__device__ __forceinline__ double bin_centre(const ParticleArgs& a, int k) {
    const double e0 = __dadd_rn(__dmul_rn((double)k, a.bc_step), a.cut_left);
    const double e1 = k + 1 >= a.S ? a.cut_right
                                   : __dadd_rn(__dmul_rn((double)(k + 1), a.bc_step), a.cut_left);
    return __dmul_rn(__dadd_rn(e0, e1), 0.5);
}

// The same for k + 1 < S (every table entry: k <= S - 2).
__device__ __forceinline__ double bin_centre_inner(const ParticleArgs& a, int k) {
    const double e0 = __dadd_rn(__dmul_rn((double)k, a.bc_step), a.cut_left);
    const double e1 = __dadd_rn(__dmul_rn((double)(k + 1), a.bc_step), a.cut_left);
    return __dmul_rn(__dadd_rn(e0, e1), 0.5);
}

template <int PREC, int TAB>
__device__ __forceinline__ typename TableEntry<PREC>::T table_at(const ParticleArgs& a,
                                                                 const void* stab, int k) {
    using TB = typename TableEntry<PREC>::T;
    if constexpr (TAB == TAB_GLOBAL) {
        return __ldg(reinterpret_cast<const TB*>(a.table) + k);
    } else if constexpr (TAB == TAB_ENTRIES || PREC == PREC_F32P64) {
        return reinterpret_cast<const TB*>(stab)[k];
    } else {
        const double* V = reinterpret_cast<const double*>(stab);
        return lik_entry0(V[k], V[k + 1], bin_centre_inner(a, k), a.charge, a.lik_inv_w);
    }
}

struct __align__(16) TurnConsts {
    double2 op[kMaxRfEngine];  // {omega_rf, phi_rf}: one 16-byte load per harmonic
    double V[kMaxRfEngine];
    float Vf[kMaxRfEngine];
    double acc;
    DriftTurn d;
};


template <int PREC, int SOLVER, bool LIK, bool KICK, bool HIST, bool WARP_AGG,
          int TAB = TAB_GLOBAL>
__device__ __forceinline__ void track_one(double& t,
                                          typename Coord<PREC>::E& e,
                                          const TurnConsts& c,
                                          const ParticleArgs& a, int* sh, int order,
                                          const void* stab = nullptr) {
    using E = typename Coord<PREC>::E;
    if (KICK) {
        if constexpr (PREC == PREC_Q32P64) {
            // the turn's whole energy change in float64, rounded once
            double inc = 0.0;
            if (LIK) {
                const double f = floor((t - a.bc0) * a.lik_inv_w);
                if (f >= 0.0 && f < (double)(a.S - 1)) {
                    const double2 tb = table_at<PREC, TAB>(a, stab, (int)f);
                    inc = __fma_rn(t, tb.x, tb.y);
                }
            }
            double s = 0.0;
            for (int j = 0; j < a.n_rf; ++j) s += c.V[j] * rf_sin(c.op[j].x * t + c.op[j].y);
            e = q32_add(e, inc + (a.charge * s + c.acc), a);
        } else {
            if (LIK) {
                const double f = floor((t - a.bc0) * a.lik_inv_w);
                if (f >= 0.0 && f < (double)(a.S - 1)) {
                    const int k = (int)f;
                    const auto tb = table_at<PREC, TAB>(a, stab, k);
                    if (PREC == PREC_F64) {
                        e = __dadd_rn(e, __fma_rn(t, tb.x, tb.y));
                    } else {
                        const float x = (float)(t - (a.bc0 + (double)k * a.bw));
                        e += __fmaf_rn(tb.y, x, tb.x);
                    }
                }
            }
            if (PREC == PREC_F64) {
                double s = 0.0;
                for (int j = 0; j < a.n_rf; ++j) s += c.V[j] * rf_sin(c.op[j].x * t + c.op[j].y);
                e += a.charge * s + c.acc;
            } else {
                float s = 0.0f;
                for (int j = 0; j < a.n_rf; ++j)
                    s += c.Vf[j] * rf_sinf(fma(c.op[j].x, t, c.op[j].y));
                e += (float)a.charge * s + (float)c.acc;
            }
        }
        // dt accumulates in float64 in every precision mode
        const double de = energy_value<PREC>(e, a);
        if (SOLVER == BLOND_SOLVER_SIMPLE)
            t = drift_simple<double>(t, de, c.d.simple);
        else if (SOLVER == BLOND_SOLVER_LEGACY)
            t = drift_legacy<double>(t, de, c.d.Tr, c.d.e0, c.d.e1, c.d.e2, order);
        else
            t = drift_exact<double>(t, de, c.d.Tr, c.d.ib2, c.d.ie2, c.d.a0, c.d.a1,
                                    c.d.a2, c.d.energy);
    }
    (void)sh;
}

// The RF voltage sum of two particles in float64, harmonic by harmonic in
// the reference's order.  RF2: two harmonics (the double-RF systems) are
// written out so that the four sines are independent instruction streams;
// the same expressions as the loop, so the same roundings.  (The batched
// pass gains 2 % from it, C3; the single-beam packed pass loses 5 %, C5.)
template <bool RF2>
__device__ __forceinline__ void rf_sum_pair(const TurnConsts& c, int n_rf, double t0,
                                            double t1, double& x0, double& x1) {
    if (RF2 && n_rf == 2) {
        const double s00 = rf_sin(c.op[0].x * t0 + c.op[0].y);
        const double s10 = rf_sin(c.op[0].x * t1 + c.op[0].y);
        const double s01 = rf_sin(c.op[1].x * t0 + c.op[1].y);
        const double s11 = rf_sin(c.op[1].x * t1 + c.op[1].y);
        x0 += c.V[0] * s00;
        x1 += c.V[0] * s10;
        x0 += c.V[1] * s01;
        x1 += c.V[1] * s11;
        return;
    }
    for (int j = 0; j < n_rf; ++j) {
        x0 += c.V[j] * rf_sin(c.op[j].x * t0 + c.op[j].y);
        x1 += c.V[j] * rf_sin(c.op[j].x * t1 + c.op[j].y);
    }
}

// Two particles at once, with the interpolation-table gathers (L2-resident,
// the longest-latency loads of the pass) issued before the RF sines so their
// latency overlaps the sine arithmetic.  Same operations, in the same order
// per particle, as two calls of track_one.
template <int PREC, int SOLVER, bool LIK, int TAB = TAB_GLOBAL, bool RF2 = false>
__device__ __forceinline__ void track_pair(double& t0, double& t1,
                                           typename Coord<PREC>::E& e0,
                                           typename Coord<PREC>::E& e1,
                                           const TurnConsts& c, const ParticleArgs& a,
                                           int order, const void* stab = nullptr) {
    using E = typename Coord<PREC>::E;
    using TB = typename TableEntry<PREC>::T;
    bool in0 = false, in1 = false;
    TB tb0, tb1;
    float x0f = 0.0f, x1f = 0.0f;  // F32P64: offsets from the slice centre
    if (LIK) {
        // floor(y) in [0, S - 2] exactly when y is in [0, S - 1); the
        // round-down conversion saturates outside the int range, so one
        // unsigned compare tests it.  (A NaN y converts to 0 and takes
        // entry 0; its particle's energy is NaN from the RF kick anyway.)
        const double y0 = (t0 - a.bc0) * a.lik_inv_w;
        const double y1 = (t1 - a.bc0) * a.lik_inv_w;
        const int r0 = __double2int_rd(y0), r1 = __double2int_rd(y1);
        in0 = (unsigned)r0 < (unsigned)(a.S - 1);
        in1 = (unsigned)r1 < (unsigned)(a.S - 1);
        const int k0 = in0 ? r0 : 0, k1 = in1 ? r1 : 0;
        tb0 = table_at<PREC, TAB>(a, stab, k0);
        tb1 = table_at<PREC, TAB>(a, stab, k1);
        if (PREC == PREC_F32P64) {
            // offsets from the slice centre, needed before t changes
            x0f = (float)(t0 - (a.bc0 + (double)k0 * a.bw));
            x1f = (float)(t1 - (a.bc0 + (double)k1 * a.bw));
        }
    }
    if constexpr (PREC == PREC_Q32P64) {
        // the turn's whole energy change in float64, rounded once per particle
        double x0 = 0.0, x1 = 0.0;
        rf_sum_pair<RF2>(c, a.n_rf, t0, t1, x0, x1);
        const double i0 = (LIK && in0) ? __fma_rn(t0, tb0.x, tb0.y) : 0.0;
        const double i1 = (LIK && in1) ? __fma_rn(t1, tb1.x, tb1.y) : 0.0;
        e0 = q32_add(e0, i0 + (a.charge * x0 + c.acc), a);
        e1 = q32_add(e1, i1 + (a.charge * x1 + c.acc), a);
    } else {
        E s0, s1;
        if (PREC == PREC_F64) {
            double x0 = 0.0, x1 = 0.0;
            rf_sum_pair<RF2>(c, a.n_rf, t0, t1, x0, x1);
            s0 = (E)x0;
            s1 = (E)x1;
        } else {
            float x0 = 0.0f, x1 = 0.0f;
            if (RF2 && a.n_rf == 2) {
                // as rf_sum_pair: four independent sines, the loop's expressions
                const float s00 = rf_sinf(fma(c.op[0].x, t0, c.op[0].y));
                const float s10 = rf_sinf(fma(c.op[0].x, t1, c.op[0].y));
                const float s01 = rf_sinf(fma(c.op[1].x, t0, c.op[1].y));
                const float s11 = rf_sinf(fma(c.op[1].x, t1, c.op[1].y));
                x0 += c.Vf[0] * s00;
                x1 += c.Vf[0] * s10;
                x0 += c.Vf[1] * s01;
                x1 += c.Vf[1] * s11;
            } else {
                // unrolled by two: C2 F32P64 (one harmonic) pass 47.3 -> 46.8 us
#pragma unroll 2
                for (int j = 0; j < a.n_rf; ++j) {
                    x0 += c.Vf[j] * rf_sinf(fma(c.op[j].x, t0, c.op[j].y));
                    x1 += c.Vf[j] * rf_sinf(fma(c.op[j].x, t1, c.op[j].y));
                }
            }
            s0 = (E)x0;
            s1 = (E)x1;
        }
        if (LIK) {
            if (PREC == PREC_F64) {
                if (in0) e0 = __dadd_rn(e0, __fma_rn(t0, tb0.x, tb0.y));
                if (in1) e1 = __dadd_rn(e1, __fma_rn(t1, tb1.x, tb1.y));
            } else {
                if (in0) e0 += __fmaf_rn(tb0.y, x0f, tb0.x);
                if (in1) e1 += __fmaf_rn(tb1.y, x1f, tb1.x);
            }
        }
        const E q = (E)a.charge, acc = (E)c.acc;
        e0 += q * s0 + acc;
        e1 += q * s1 + acc;
    }
    const double d0 = energy_value<PREC>(e0, a), d1 = energy_value<PREC>(e1, a);
    if (SOLVER == BLOND_SOLVER_SIMPLE) {
        t0 = drift_simple<double>(t0, d0, c.d.simple);
        t1 = drift_simple<double>(t1, d1, c.d.simple);
    } else if (SOLVER == BLOND_SOLVER_LEGACY) {
        t0 = drift_legacy<double>(t0, d0, c.d.Tr, c.d.e0, c.d.e1, c.d.e2, order);
        t1 = drift_legacy<double>(t1, d1, c.d.Tr, c.d.e0, c.d.e1, c.d.e2, order);
    } else {
        t0 = drift_exact<double>(t0, d0, c.d.Tr, c.d.ib2, c.d.ie2, c.d.a0, c.d.a1,
                                 c.d.a2, c.d.energy);
        t1 = drift_exact<double>(t1, d1, c.d.Tr, c.d.ib2, c.d.ie2, c.d.a0, c.d.a1,
                                 c.d.a2, c.d.energy);
    }
}

__device__ __forceinline__ int engine_bin(double t, double cut_left, double inv_w, int S) {
    // floor(y) in [0, S) exactly when y is in [0, S); the round-down
    // conversion saturates outside the int range and gives 0 for NaN,
    // which the y == y test excludes
    const double y = __dmul_rn(__dsub_rn(t, cut_left), inv_w);
    const int k = __double2int_rd(y);
    return ((unsigned)k < (unsigned)S && y == y) ? k : -1;
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
    // one atomic for either half; the wrap test and its carries are the
    // rare branch
    const bool lo = b < half;
    const int w = lo ? b : b - half;
    const unsigned old = atomicAdd(&sh[w], lo ? 1u : 0x10000u);
    if ((lo ? (old & 0xffffu) : (old >> 16)) == 0xffffu) {
        atomicAdd(&gh[b], 65536);
        if (lo) {
            if ((old >> 16) == 0xffffu) atomicAdd(&gh[b + half], 65536);
            const unsigned o2 = atomicSub(&sh[b], 0x10000u);
            if ((o2 >> 16) == 0u) atomicAdd(&gh[b + half], -65536);
        }
    }
}

// Packed deposit while no counter can wrap (the block has deposited at
// most 65535 particles since its counters were zero): no returned value,
// no test.
__device__ __forceinline__ void deposit_packed_nowrap(unsigned* sh, int half, int b) {
    if (b < 0) return;
    const bool lo = b < half;
    atomicAdd(&sh[lo ? b : b - half], lo ? 1u : 0x10000u);
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
__device__ __forceinline__ void stream_store(int2* p, int2 v, uint64_t pol) {
    asm volatile("st.global.L2::cache_hint.v2.s32 [%0], {%1, %2}, %3;" ::"l"(p), "r"(v.x),
                 "r"(v.y), "l"(pol) : "memory");
}
__device__ __forceinline__ void stream_store(int* p, int v, uint64_t pol) {
    asm volatile("st.global.L2::cache_hint.s32 [%0], %1, %2;" ::"l"(p), "r"(v), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ int2 stream_load(const int2* p, uint64_t pol) {
    int2 v;
    asm volatile("ld.global.L2::cache_hint.v2.s32 {%0, %1}, [%2], %3;"
                 : "=r"(v.x), "=r"(v.y) : "l"(p), "l"(pol) : "memory");
    return v;
}
__device__ __forceinline__ int stream_load(const int* p, uint64_t pol) {
    int v;
    asm volatile("ld.global.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol)
                 : "memory");
    return v;
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
            c.op[j] = make_double2(a.om[t_idx * a.n_rf + j], a.ph[t_idx * a.n_rf + j]);
        }
        if (threadIdx.x == 0) {
            c.acc = a.interp ? 0.0 : a.acc[t_idx];
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
            if (!a.no_deposit) {
                deposit(hd, b0, WARP_AGG, 0xffffffffu);
                deposit(hd, b1, WARP_AGG, 0xffffffffu);
            }
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
            if (!a.no_deposit) {
                deposit(hd, b0, WARP_AGG, 0xffffffffu);
                deposit(hd, b1, WARP_AGG, 0xffffffffu);
            }
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
        if (b >= 0 && !a.no_deposit) atomicAdd(&hd[b], 1);
    }
    if (!a.global_hist) cluster_flush(sh, a.hist, a.S);
}

// ------------------------------------------------- shared-table plain pass
// The plain pass with the induced kick's table in shared memory.  F64 and
// Q32P64 keep only the induced voltage (8 B per slice: 128 KB at 2^14
// slices, where the {slope, offset} table is 256 KB); each particle forms
// its entry with lik_entry from V_k, V_{k+1} and the bin centre, which gives
// the head's table entry bit for bit.  F32P64 keeps the float2 table.  A
// gather then costs a shared-memory access instead of an L2 round trip --
// the global-table pass's top stall (long scoreboard on the table loads,
// L1 hit rate ~25 %).  One 1024-thread block per SM holds the table, the
// packed 16-bit block histogram (deposit_packed, exact under wraps) and the
// prefetch ring; the block copies the table after the head has completed.
__device__ __forceinline__ void copy16_async(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void copy8_async(void* smem, const void* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(
                     (uint32_t)__cvta_generic_to_shared(smem)), "l"(gmem) : "memory");
}

// Bytes of the shared table (before padding to 16) for S slices.
template <int PREC>
__host__ __device__ constexpr size_t stab_table_bytes(int S) {
    return PREC == PREC_F32P64 ? (size_t)(S - 1) * 8 : (size_t)S * 8;
}
__host__ __device__ constexpr size_t pad16(size_t x) { return (x + 15) & ~(size_t)15; }

// TAB = TAB_GLOBAL gives the same pass over the global table (no copy):
// the plain pass with a packed histogram, which fits 2^16-slice profiles
// beside the ring.
template <int PREC, int SOLVER, int NST, int TAB = TAB_SHARED>
__global__ void __launch_bounds__(kEngineThreads, 1)
particle_kernel_stab(const ParticleArgs a) {
    using E = typename Coord<PREC>::E;
    using E2 = typename Vec2<E>::type;
    extern __shared__ __align__(16) unsigned char dsm[];
    __shared__ TurnConsts c;
    pdl_launch_dependents();
    const int S = a.S;
    const int half = (S + 1) / 2;
    const size_t tbytes = TAB == TAB_SHARED ? stab_table_bytes<PREC>(S) : 0;
    const size_t tpad = pad16(tbytes), hpad = pad16((size_t)half * 4);
    const void* stab = dsm;
    unsigned* sh = reinterpret_cast<unsigned*>(dsm + tpad);
    for (int k = threadIdx.x; k < half; k += blockDim.x) sh[k] = 0u;
    pdl_wait();  // the head's table / voltage, counter and cleared histogram
    long long t_idx = a.turn ? (*a.turn - 1) : 0;
    if (t_idx < 0) t_idx = 0;
    if (t_idx >= a.n_turns) t_idx = a.n_turns - 1;
    for (int j = threadIdx.x; j < a.n_rf; j += blockDim.x) {
        c.V[j] = a.V[t_idx * a.n_rf + j];
        c.Vf[j] = (float)c.V[j];
        c.op[j] = make_double2(a.om[t_idx * a.n_rf + j], a.ph[t_idx * a.n_rf + j]);
    }
    if (threadIdx.x == 0) {
        c.acc = a.interp ? 0.0 : a.acc[t_idx];
        c.d = a.drift[t_idx + 1];
    }
    // the table (L2-resident): 16-byte asynchronous copies, one group
    // (empty for the global-table form)
    if (TAB == TAB_SHARED) {
        const char* src = reinterpret_cast<const char*>(PREC == PREC_F32P64 ? a.table
                                                                            : (const void*)a.vind);
        const size_t n16 = tbytes / 16;
        for (size_t q = threadIdx.x; q < n16; q += blockDim.x) copy16_async(dsm + 16 * q, src + 16 * q);
        if (threadIdx.x == 0 && (tbytes & 15))
            *reinterpret_cast<double*>(dsm + 16 * n16) =
                *reinterpret_cast<const double*>(src + 16 * n16);
        ring_commit();
    } else {
        ring_commit();
    }
    double* dt = reinterpret_cast<double*>(a.dt);
    E* dE = reinterpret_cast<E*>(a.dE);
    const int64_t npairs = a.n / 2;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int order = a.order;
    const int lane = threadIdx.x & 31;
    int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31);
    const uint64_t pol = evict_first_policy();
    // The block deposits at most 2 x blockDim particles an iteration, so for
    // its first `safe` iterations (<= 65535 deposits) no counter can wrap
    // and the deposits skip the wrap test; a barrier separates them from
    // the tested ones (warps are not in step inside the loop).  Ring
    // variants only.
    const int safe = 65535 / (2 * (int)blockDim.x);
    auto deposit2 = [&](int b0, int b1, auto tested) {
        if constexpr (decltype(tested)::value) {
            deposit_packed(sh, half, a.hist, b0);
            deposit_packed(sh, half, a.hist, b1);
        } else {
            deposit_packed_nowrap(sh, half, b0);
            deposit_packed_nowrap(sh, half, b1);
        }
    };
    if (NST == 0) {
        ring_wait<0>();
        __syncthreads();  // every thread's part of the table has landed
        auto step = [&](auto tested) {
            const int64_t p = base + lane;
            int b0 = -1, b1 = -1;
            if (p < npairs) {
                double2 tt = stream_load(reinterpret_cast<const double2*>(dt) + p, pol);
                E2 ee = stream_load(reinterpret_cast<const E2*>(dE) + p, pol);
                track_pair<PREC, SOLVER, true, TAB>(tt.x, tt.y, ee.x, ee.y, c, a, order, stab);
                stream_store(reinterpret_cast<double2*>(dt) + p, tt, pol);
                stream_store(reinterpret_cast<E2*>(dE) + p, ee, pol);
                b0 = engine_bin(tt.x, a.cut_left, a.inv_w, S);
                b1 = engine_bin(tt.y, a.cut_left, a.inv_w, S);
            }
            deposit2(b0, b1, tested);
        };
        // (without the ring the split loop measured slower at 2^16 slices)
        for (; base < npairs; base += stride) step(std::true_type{});
    } else {
        double2* rdt = reinterpret_cast<double2*>(dsm + tpad + hpad);
        E2* rdE = reinterpret_cast<E2*>(rdt + (size_t)NST * blockDim.x);
        const double2* gdt = reinterpret_cast<const double2*>(dt);
        const E2* gdE = reinterpret_cast<const E2*>(dE);
        auto fill = [&](int slot, int64_t p) {
            if (p < npairs) {
                ring_copy16(&rdt[slot * blockDim.x + threadIdx.x], &gdt[p], pol);
                if (sizeof(E2) == 16) ring_copy16(&rdE[slot * blockDim.x + threadIdx.x], &gdE[p], pol);
                else ring_copy8(&rdE[slot * blockDim.x + threadIdx.x], &gdE[p], pol);
            }
            ring_commit();
        };
#pragma unroll
        for (int s = 0; s < NST - 1; ++s) fill(s, base + s * stride + lane);
        // groups complete in order: the table's (the oldest) has landed
        ring_wait<NST - 1>();
        __syncthreads();
        int slot = 0;
        auto step = [&](auto tested) {
            fill(slot == 0 ? NST - 1 : slot - 1, base + (NST - 1) * stride + lane);
            if (a.l2_ahead && threadIdx.x == 0) {
                const int64_t pb = base + (int64_t)NST * stride;
                if (pb < npairs) {
                    const int64_t cnt = min((int64_t)blockDim.x, npairs - pb);
                    if (((uintptr_t)(gdt + pb) & 15) == 0)
                        l2_prefetch(gdt + pb, (uint32_t)(cnt * 16), pol);
                    if (((uintptr_t)(gdE + pb) & 15) == 0 && ((cnt * sizeof(E2)) & ~(int64_t)15))
                        l2_prefetch(gdE + pb, (uint32_t)((cnt * sizeof(E2)) & ~(int64_t)15), pol);
                }
            }
            ring_wait<NST - 1>();
            const int64_t p = base + lane;
            int b0 = -1, b1 = -1;
            if (p < npairs) {
                double2 tt = rdt[slot * blockDim.x + threadIdx.x];
                E2 ee = rdE[slot * blockDim.x + threadIdx.x];
                track_pair<PREC, SOLVER, true, TAB>(tt.x, tt.y, ee.x, ee.y, c, a, order, stab);
                stream_store(reinterpret_cast<double2*>(dt) + p, tt, pol);
                stream_store(reinterpret_cast<E2*>(dE) + p, ee, pol);
                b0 = engine_bin(tt.x, a.cut_left, a.inv_w, S);
                b1 = engine_bin(tt.y, a.cut_left, a.inv_w, S);
            }
            deposit2(b0, b1, tested);
            slot = slot + 1 == NST ? 0 : slot + 1;
        };
        int it = 0;
        for (; base < npairs && it < safe; base += stride, ++it) step(std::false_type{});
        __syncthreads();
        for (; base < npairs; base += stride) step(std::true_type{});
        ring_wait<0>();
    }
    // odd tail particle
    if ((a.n & 1) && blockIdx.x == 0 && threadIdx.x == 0) {
        double t = dt[a.n - 1];
        E e = dE[a.n - 1];
        track_one<PREC, SOLVER, true, true, true, false, TAB>(t, e, c, a, nullptr, order, stab);
        dt[a.n - 1] = t;
        dE[a.n - 1] = e;
        deposit_packed(sh, half, a.hist, engine_bin(t, a.cut_left, a.inv_w, S));
    }
    __syncthreads();
    for (int k = threadIdx.x; k < half; k += blockDim.x) {
        const unsigned v = sh[k];
        if (v & 0xffffu) atomicAdd(&a.hist[k], (int)(v & 0xffffu));
        if ((v >> 16) && k + half < S) atomicAdd(&a.hist[k + half], (int)(v >> 16));
    }
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
    if ((threadIdx.x & 31) == 0) atomicOr(err, ERR_WAIT);
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
        c.op[j] = make_double2(a.om[t_idx * a.n_rf + j], a.ph[t_idx * a.n_rf + j]);
    }
    if (threadIdx.x == 0) {
        c.acc = a.interp ? 0.0 : a.acc[t_idx];
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
                if (!a.no_deposit) {
                    block_deposit<HIST>(sh, half, a.hist,
                                        engine_bin(tt.x, a.cut_left, a.inv_w, a.S));
                    block_deposit<HIST>(sh, half, a.hist,
                                        engine_bin(tt.y, a.cut_left, a.inv_w, a.S));
                }
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
            const int b = a.no_deposit ? -1 : engine_bin(t, a.cut_left, a.inv_w, a.S);
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
static __global__ void profile_kernel(int* hist, double* profile, int S, int clear,
                               long long* turn) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < S;
         k += gridDim.x * blockDim.x) {
        profile[k] = (double)hist[k];
        if (clear) hist[k] = 0;
    }
    if (clear && turn && blockIdx.x == 0 && threadIdx.x == 0) *turn += 1;
}

}  // namespace bb

namespace bb {

static void free_ptr(void* p) {
    if (p) cudaFree(p);
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

static int upload(void** dst, const void* src, size_t bytes) {
    free_ptr(*dst);
    *dst = nullptr;
    BB_CUDA(cudaMalloc(dst, bytes));
    BB_CUDA(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
    return BLOND_OK;
}

}  // namespace bb
