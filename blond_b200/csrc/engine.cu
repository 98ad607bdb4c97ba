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
#include "engine_device.cuh"

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
    // the bin centres are numpy.linspace midpoints of the cuts, bit for bit
    // (the shared-table pass recomputes them)
    bool bc_linspace = false;
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
    double lsb = 0.0;  // Q32P64: eV per count of dE (blond_engine_set_energy_unit)
    // interpolated tracker (blond_engine_set_interpolation): RF + induced
    // voltage interpolated from the table, no separate RF kick
    bool interp = false;
    // smooth slicing (blond_engine_set_smooth): fixed-point accumulator,
    // its bits per particle and the last-block ticket
    bool smooth = false;
    long long* d_acc64 = nullptr;
    int* d_smooth_ticket = nullptr;
    int smooth_bits = 0;
    // tuning
    int threads = 512;
    int blocks_per_sm = 2;
    int turns_per_graph = 50;
    int variant = 0;  // 0: TMA-pipelined particle pass, 1: plain loads,
                      // 2: plain loads with the table in shared memory,
                      // 3: plain loads, packed histogram, global table
    int hist_mode = -1;  // -1 automatic, else HIST_AGG/I32/PACKED/GLOBAL
    int ring = 0;        // plain pass: prefetch ring stages (0 = direct loads)
    int cluster = 1;     // plain pass: blocks whose histograms merge on chip
    bool l2_ahead = false;  // shared-table pass: L2 prefetch beyond the ring
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

// Dynamic shared memory of the shared-table pass (table, packed histogram,
// ring), or -1 when the pass does not apply: it needs the head's induced
// voltage alone as the table source (an FFT impedance, no interpolated RF
// voltage), integer deposits, linspace bin centres, and room for it all.
template <int PREC>
static int stab_smem(const blond_engine* e, int ring) {
    if (!e->has_fft || e->interp || e->smooth || !e->bc_linspace) return -1;
    const size_t bytes = pad16(stab_table_bytes<PREC>(e->S)) +
                         pad16((size_t)((e->S + 1) / 2) * 4) +
                         (size_t)ring * kEngineThreads * ring_bytes<PREC>();
    const size_t limit = (size_t)device_info().max_smem_optin - sizeof(TurnConsts) - 1024;
    return bytes <= limit ? (int)bytes : -1;
}

// Dynamic shared memory of the packed plain pass over the global table
// (variant 3: packed histogram + ring), or -1 when it does not fit or the
// turn deposits no integer counts.
template <int PREC>
static int packed_smem(const blond_engine* e, int ring) {
    if (e->smooth) return -1;
    const size_t bytes = pad16((size_t)((e->S + 1) / 2) * 4) +
                         (size_t)ring * kEngineThreads * ring_bytes<PREC>();
    const size_t limit = (size_t)device_info().max_smem_optin - sizeof(TurnConsts) - 1024;
    return bytes <= limit ? (int)bytes : -1;
}

template <int PREC, int SOLVER, int TAB, int NST>
static auto packed_kernel() {
    return particle_kernel_stab<PREC, SOLVER, NST, TAB>;
}

template <int PREC, int SOLVER>
static int launch_stab(blond_engine* e, const ParticleArgs& a, cudaStream_t s, bool launch) {
    const bool shared = e->variant == 2;
    const int ring = shared ? (e->ring ? 2 : 0) : (e->ring >= 4 ? 4 : (e->ring ? 2 : 0));
    const int smem = shared ? stab_smem<PREC>(e, ring) : packed_smem<PREC>(e, ring);
    if (smem < 0) {
        set_error(shared ? "engine: the shared-table pass does not apply to this engine"
                         : "engine: the packed-histogram pass does not fit this engine");
        return BLOND_ERR_UNSUPPORTED;
    }
    auto k = shared ? (ring ? packed_kernel<PREC, SOLVER, TAB_SHARED, 2>()
                            : packed_kernel<PREC, SOLVER, TAB_SHARED, 0>())
                    : (ring == 4 ? packed_kernel<PREC, SOLVER, TAB_GLOBAL, 4>()
                       : ring ? packed_kernel<PREC, SOLVER, TAB_GLOBAL, 2>()
                              : packed_kernel<PREC, SOLVER, TAB_GLOBAL, 0>());
    int rc;
    if ((rc = allow_smem_once(k))) return rc;
    if (launch) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(device_info().sm_count, 1, 1);
        cfg.blockDim = dim3(kEngineThreads, 1, 1);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        int na = 0;
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

template <int PREC, int SOLVER, bool LIK, bool KICK>
static int launch_particles_t(blond_engine* e, const ParticleArgs& a, cudaStream_t s,
                              bool launch) {
    if constexpr (KICK) {
        if (e->variant == 2 || e->variant == 3) {
            if constexpr (LIK) {
                return launch_stab<PREC, SOLVER>(e, a, s, launch);
            } else {
                set_error(e->variant == 2
                              ? "engine: the shared-table pass does not apply to this engine "
                                "(no interpolated kick)"
                              : "engine: the packed-histogram pass does not apply to this "
                                "engine (no interpolated kick)");
                return BLOND_ERR_UNSUPPORTED;
            }
        }
    }
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
    // the interpolated tracker kicks through the table even without impedance
    const bool lik = e->has_fft || e->has_ind || e->interp;
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
    a.lsb = e->lsb;
    a.inv_lsb = e->lsb > 0 ? 1.0 / e->lsb : 0.0;
    a.err = e->d_err;
    if (e->interp) {
        a.n_rf = 0;
        a.interp = 1;
    }
    a.no_deposit = e->smooth ? 1 : 0;
    a.vind = e->d_vind;
    a.l2_ahead = e->l2_ahead ? 1 : 0;
    a.cut_right = e->cut_right;
    a.bc_step = (e->cut_right - e->cut_left) / (double)e->S;
    return a;
}

static int launch_particles_a(blond_engine* e, const ParticleArgs& a, bool kick,
                              cudaStream_t s, bool launch) {
    switch (e->precision) {
        case BLOND_PREC_F64: return launch_particles_p<PREC_F64>(e, a, kick, s, launch);
        case BLOND_PREC_F32P64: return launch_particles_p<PREC_F32P64>(e, a, kick, s, launch);
        default: return launch_particles_p<PREC_Q32P64>(e, a, kick, s, launch);
    }
}

static int launch_particles(blond_engine* e, bool kick, cudaStream_t s,
                            bool launch = true) {
    return launch_particles_a(e, particle_args(e), kick, s, launch);
}

// Bytes of one stored energy: float64 (F64), float32 (F32P64), int32 (Q32P64).
static size_t energy_bytes(int precision) {
    return precision == BLOND_PREC_F64 ? sizeof(double) : 4;
}

// The particle pass over particles [off, off + cnt) of the bound beam (off
// even, so pairs stay 16-byte aligned); deposits into the same histogram.
static int launch_particles_range(blond_engine* e, int64_t off, int64_t cnt,
                                  cudaStream_t s) {
    ParticleArgs a = particle_args(e);
    a.dt = static_cast<double*>(e->dt) + off;
    a.dE = static_cast<char*>(e->dE) + energy_bytes(e->precision) * (size_t)off;
    a.n = cnt;
    return launch_particles_a(e, a, true, s, true);
}

// Smooth slicing inside the fused turn (Profile with smooth=True,
// profile.py:764-773), the weights of histogram.cpp:75-132 (bin k gets
// 0.5 - d, which may be negative, its neighbour 0.5 + d).  Each weight is
// rounded to a multiple of 2^-bits and accumulated with 64-bit integer
// atomics -- in shared memory when the profile fits, then into the global
// accumulator -- so the sum does not depend on the order of the atomics and
// every run gives the same bits.  bits = min(52, 62 - ceil(log2(1.5 n + 2)))
// keeps |sum| below 2^62.  The block that takes the last ticket converts the
// accumulator into the float64 profile and zeroes it.
constexpr int kSmoothThreads = 512;

__global__ void __launch_bounds__(kSmoothThreads)
smooth_deposit_kernel(const double* __restrict__ dt, int64_t n, double cut_left, double inv_w,
                      double lo, double hi, int S, int bits, int use_smem,
                      unsigned long long* __restrict__ acc, double* __restrict__ profile,
                      int* __restrict__ ticket) {
    extern __shared__ unsigned long long sacc[];
    if (use_smem) {
        for (int k = threadIdx.x; k < S; k += blockDim.x) sacc[k] = 0ull;
        __syncthreads();
    }
    unsigned long long* dst = use_smem ? sacc : acc;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        int k, k2;
        double w1 = 0.0, w2 = 0.0;
        smooth_weights<double>(dt[i], cut_left, inv_w, lo, hi, S, k, k2, w1, w2);
        if (k >= 0) atomicAdd(&dst[k], (unsigned long long)llrint(ldexp(w1, bits)));
        if (k2 >= 0) atomicAdd(&dst[k2], (unsigned long long)llrint(ldexp(w2, bits)));
    }
    __shared__ bool last;
    __syncthreads();
    if (use_smem)
        for (int k = threadIdx.x; k < S; k += blockDim.x)
            if (sacc[k]) atomicAdd(&acc[k], sacc[k]);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1) == (int)gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int k = threadIdx.x; k < S; k += blockDim.x) {
        const long long v = (long long)atomicExch(&acc[k], 0ull);
        profile[k] = ldexp((double)v, -bits);
    }
    if (threadIdx.x == 0) *ticket = 0;
}

static int smooth_bits_for(int64_t n) {
    int lg = 0;
    while (lg < 62 && (1ll << lg) < 3 * n / 2 + 2) ++lg;
    return std::min(52, 62 - lg);
}

static int launch_smooth_deposit(blond_engine* e, cudaStream_t s) {
    const double w = (e->cut_right - e->cut_left) / e->S;
    const double lo = e->cut_left + w * 0.5, hi = e->cut_right - w * 0.5;
    const int limit = device_info().max_smem_optin - 1024;
    const size_t smem = sizeof(unsigned long long) * (size_t)e->S;
    const bool use_smem = (int64_t)smem <= limit;
    static std::mutex mu;
    static std::set<int> done;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (!done.count(device_info().device)) {
            BB_CUDA(cudaFuncSetAttribute(smooth_deposit_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, limit));
            done.insert(device_info().device);
        }
    }
    const int grid = particle_grid(e->n, kSmoothThreads, use_smem && smem > 96 * 1024 ? 1 : 2);
    smooth_deposit_kernel<<<grid, kSmoothThreads, use_smem ? smem : 0, s>>>(
        static_cast<const double*>(e->dt), e->n, e->cut_left, e->inv_w, lo, hi, e->S,
        e->smooth_bits, use_smem ? 1 : 0, reinterpret_cast<unsigned long long*>(e->d_acc64),
        e->d_profile, e->d_smooth_ticket);
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

static int launch_profile(blond_engine* e, bool clear, cudaStream_t s) {
    // smooth slicing: the deposit pass wrote the profile; the head only
    // advances the turn counter
    if (e->smooth) {
        if (clear) {
            profile_kernel<<<1, 32, 0, s>>>(e->d_hist, e->d_profile, 0, 1, e->d_turn);
            BB_LAUNCH_CHECK();
        }
        return BLOND_OK;
    }
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

// The interpolated tracker's table (tracker.py:586-601): the RF voltage at
// the bin centres (rf_volt_comp, kick.cpp:37-51) plus the induced voltage
// (vind, when there is an impedance: the head wrote it), with the turn's
// acceleration kick in the offsets (linear_interp_kick.cpp:44-47).  Without
// an impedance this kernel is the whole head: it also converts (and clears)
// the histogram and advances the turn counter -- then it runs as one CTA,
// so every thread reads the counter before thread 0 moves it.  After a
// spectral head (which advanced the counter) it reads turn - 1.
__global__ void __launch_bounds__(1024)
interp_table_kernel(int* hist, double* profile, int S, long long* turn_p, int head,
                    const double* V, const double* om, const double* ph, int n_rf,
                    const double* acc, const double* bc, const double* vind, double charge,
                    double inv_w, void* table, int table_f32, long long n_turns) {
    long long turn = *turn_p - (head ? 0 : 1);
    if (turn < 0) turn = 0;
    if (turn >= n_turns) turn = n_turns - 1;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    if (head)
        for (int k = tid; k < S; k += nth) {
            profile[k] = (double)hist[k];
            hist[k] = 0;
        }
    const double* Vt = V + turn * n_rf;
    const double* omt = om + turn * n_rf;
    const double* pht = ph + turn * n_rf;
    const double acc_t = acc[turn];
    auto total = [&](int k) {
        double s = 0.0;
        for (int j = 0; j < n_rf; ++j) s += Vt[j] * rf_sin(omt[j] * bc[k] + pht[j]);
        return vind ? s + vind[k] : s;  // rf_voltage + induced_voltage
    };
    for (int n = tid; n < S - 1; n += nth) {
        const double a0 = total(n), a1 = total(n + 1);
        if (!table_f32) {
            reinterpret_cast<double2*>(table)[n] = lik_entry(a0, a1, bc[n], charge, inv_w, acc_t);
        } else {
            reinterpret_cast<float2*>(table)[n] =
                make_float2((float)(charge * a0 + acc_t), (float)(charge * (a1 - a0) * inv_w));
        }
    }
    if (head) {
        __syncthreads();
        if (threadIdx.x == 0) *turn_p = *turn_p + 1;
    }
}

static int launch_interp_table(blond_engine* e, cudaStream_t s, bool head) {
    const int grid = head ? 1 : std::min(device_info().sm_count, (e->S + 255) / 256);
    interp_table_kernel<<<grid, head ? 1024 : 256, 0, s>>>(
        e->d_hist, e->d_profile, e->S, e->d_turn, head ? 1 : 0, e->d_V, e->d_om, e->d_ph,
        e->n_rf, e->d_acc, e->d_bc, head ? nullptr : e->d_vind, e->charge, e->lik_inv_w,
        e->d_table, e->precision == BLOND_PREC_F32P64 ? 1 : 0, e->n_turns);
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

static int launch_spectral_head(blond_engine* e, cudaStream_t s, bool loop) {
    if (!(e->has_fft || e->has_ind)) {
        if (!e->interp) return launch_profile(e, true, s);
        return launch_interp_table(e, s, true);
    }
    if (!e->has_fft) {
        set_error("engine: an inductive impedance needs an FFT impedance in this build");
        return BLOND_ERR_UNSUPPORTED;
    }
    SpecParams P = {};
    P.p = e->plan;
    P.mode = SPEC_FORWARD | SPEC_MULTIPLY | SPEC_INVERSE;
    P.pdl = e->pdl ? 1 : 0;
    P.n_in = e->S;
    P.profile_out = e->d_profile;
    if (e->smooth)
        P.in_f64 = e->d_profile;  // the smooth deposit's profile (read only)
    else
        P.in_i32 = e->d_hist;
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
    // the interpolated tracker's table (RF + induced voltage) follows the head
    if (e->interp) P.table = nullptr;
    // the shared-table pass forms FP64 / Q32P64 entries from the voltage
    // itself: no table to write (the beam-phase loop's SPS_RL average reads
    // it, so it stays with a loop)
    if (e->variant == 2 && e->precision != BLOND_PREC_F32P64 && !e->has_fb) P.table = nullptr;
    int rc;
    if (loop) {
        SpecLoop L;
        L.ticket = e->d_fb_ticket;
        L.fb = fb_args(e);
        rc = launch_spectral_loop(P, L, s);
    } else {
        rc = launch_spectral(P, s);
    }
    if (rc || !e->interp) return rc;
    return launch_interp_table(e, s, false);
}

static int launch_turn(blond_engine* e, cudaStream_t s) {
    int rc = launch_head(e, s);
    if (rc) return rc;
    if ((rc = launch_particles(e, true, s))) return rc;
    return e->smooth ? launch_smooth_deposit(e, s) : BLOND_OK;
}

static int check_ready(blond_engine* e) {
    if (!e->rf_set || !e->drift_set || !e->slicing_set || !e->dt) {
        set_error("engine: set_rf, set_drift, set_slicing and bind_beam must all be "
                  "called before tracking");
        return BLOND_ERR_STATE;
    }
    if (e->precision == BLOND_PREC_Q32P64 && !(e->lsb > 0)) {
        set_error("engine: precision Q32P64 needs set_energy_unit before tracking");
        return BLOND_ERR_STATE;
    }
    return BLOND_OK;
}


}  // namespace bb

extern "C" {

int blond_engine_create(blond_engine** out, int precision, int n_rf, int solver,
                        int n_slices) {
    BB_CHECK_ARG(out, "engine_create: null output");
    BB_CHECK_ARG(precision == BLOND_PREC_F64 || precision == BLOND_PREC_F32P64 ||
                     precision == BLOND_PREC_Q32P64,
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
                    (void*)e->d_vind, e->d_table, (void*)e->d_acc64,
                    (void*)e->d_smooth_ticket})
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
    e->bc_linspace = true;
    for (int k = 0; k < S && e->bc_linspace; ++k)
        e->bc_linspace = bc[k] == linspace_centre(cut_left, cut_right, S, k);
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
    e->smooth_bits = smooth_bits_for(n);
    e->graph_dirty = true;
    return BLOND_OK;
}

int blond_engine_set_interpolation(blond_engine* e, int on) {
    BB_CHECK_ARG(e, "engine_set_interpolation: null engine");
    if (on && e->has_fb && (e->fb.machine == BLOND_FB_SPS_RL || !e->has_fft)) {
        set_error("engine_set_interpolation: not with the SPS_RL loop or a beam-phase loop "
                  "without an FFT impedance");
        return BLOND_ERR_UNSUPPORTED;
    }
    e->interp = on != 0;
    e->graph_dirty = true;
    return BLOND_OK;
}

int blond_engine_set_smooth(blond_engine* e, int on) {
    BB_CHECK_ARG(e, "engine_set_smooth: null engine");
    if (on && (e->has_fb || e->d_hist != e->own_hist)) {
        set_error("engine_set_smooth: smooth slicing is not built with a beam-phase loop or "
                  "a caller-bound (sharded) histogram");
        return BLOND_ERR_UNSUPPORTED;
    }
    if (on && !e->d_acc64) {
        BB_CUDA(cudaMalloc((void**)&e->d_acc64, sizeof(long long) * (size_t)e->S));
        BB_CUDA(cudaMemset(e->d_acc64, 0, sizeof(long long) * (size_t)e->S));
        BB_CUDA(cudaMalloc((void**)&e->d_smooth_ticket, sizeof(int)));
        BB_CUDA(cudaMemset(e->d_smooth_ticket, 0, sizeof(int)));
    }
    e->smooth = on != 0;
    e->graph_dirty = true;
    return BLOND_OK;
}

int blond_engine_set_energy_unit(blond_engine* e, double lsb) {
    BB_CHECK_ARG(e, "engine_set_energy_unit: null engine");
    BB_CHECK_ARG(std::isfinite(lsb) && lsb > 0, "engine_set_energy_unit: the unit must be a "
                 "finite energy > 0 (eV per count)");
    e->lsb = lsb;
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
    if (e->smooth) return launch_smooth_deposit(e, s);
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
    if (e->smooth) {
        set_error("engine_step: the step-by-step (sharded) turn deposits integer counts; "
                  "smooth slicing runs through blond_engine_run");
        return BLOND_ERR_UNSUPPORTED;
    }
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
    BB_CHECK_ARG(e && variant >= 0 && variant <= 3,
                 "engine_set_kernel: variant 0 (staged), 1 (plain), 2 (shared table) or 3 "
                 "(plain with a packed histogram)");
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
        if (flag & ERR_WAIT) {
            set_error("engine: a bounded device-side wait gave up (bulk copy never "
                      "completed); the coordinates of this run are not valid");
            return BLOND_ERR_TIMEOUT;
        }
        set_error("engine: an energy left the 32-bit fixed-point grid (more than 2^31 - 1 "
                  "units of %g eV from 0); track again with a larger energy unit", e->lsb);
        return BLOND_ERR_RANGE;
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

int blond_engine_set_l2_prefetch(blond_engine* e, int on) {
    BB_CHECK_ARG(e, "engine_set_l2_prefetch: null engine");
    e->l2_ahead = on != 0;
    e->graph_dirty = true;
    return BLOND_OK;
}

int blond_engine_set_overlap(blond_engine* e, int on) {
    BB_CHECK_ARG(e, "engine_set_overlap: null engine");
    e->pdl = on != 0;
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
}  // extern "C"

namespace bb {

// Whole turns (head + particle pass, as tracking runs them) replayed from a
// graph of `turns` turns: one untimed replay, then `reps` timed; returns
// the milliseconds per turn.  Advances the beam and the turn counter.
static int time_graph_turns(blond_engine* e, cudaStream_t s, int turns, int reps, double* ms) {
    int rc;
    if ((rc = launch_particles(e, true, s, false))) return rc;
    if (e->has_fft && (rc = prepare_spectral())) return rc;
    cudaGraph_t g = nullptr;
    BB_CUDA(cudaStreamBeginCapture(e->cap_stream, cudaStreamCaptureModeThreadLocal));
    int lrc = BLOND_OK;
    for (int i = 0; i < turns && lrc == BLOND_OK; ++i) lrc = launch_turn(e, e->cap_stream);
    cudaError_t ce = cudaStreamEndCapture(e->cap_stream, &g);
    if (lrc || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        if (lrc) return lrc;
        set_error("engine_autotune: graph capture failed: %s", cudaGetErrorString(ce));
        return BLOND_ERR_CUDA;
    }
    cudaGraphExec_t x = nullptr;
    ce = cudaGraphInstantiate(&x, g, 0);
    cudaGraphDestroy(g);
    if (ce != cudaSuccess) {
        set_error("engine_autotune: graph instantiation failed: %s", cudaGetErrorString(ce));
        return BLOND_ERR_CUDA;
    }
    cudaEvent_t a = nullptr, b = nullptr;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaGraphLaunch(x, s);
    cudaEventRecord(a, s);
    for (int r = 0; r < reps; ++r) cudaGraphLaunch(x, s);
    cudaEventRecord(b, s);
    ce = cudaEventSynchronize(b);
    float t = 0.f;
    if (ce == cudaSuccess) cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaGraphExecDestroy(x);
    if (ce != cudaSuccess) {
        set_error("engine_autotune: %s", cudaGetErrorString(ce));
        return BLOND_ERR_CUDA;
    }
    *ms = (double)t / ((double)turns * reps);
    return BLOND_OK;
}

// Programmatic dependent launch on or off, whichever replays whole turns
// faster with the chosen particle pass (the early launch of the next
// kernel pays at short profiles and costs at long ones).  Each setting
// starts from the same snapshot of the turn counter, induced voltage and
// profile, which are put back afterwards; the caller restores the beam and
// histogram.  Skipped (overlap left as it is) with a beam-phase loop or
// smooth slicing, whose turn state is not snapshotted, and when fewer
// turns than it needs are left in the programme.
static int tune_overlap(blond_engine* e, cudaStream_t s, const void* sdt, const void* sdE,
                        const int* shist, int* chosen) {
    constexpr int kTurns = 4, kReps = 3;
    *chosen = e->pdl ? 1 : 0;
    if (e->has_fb || e->smooth || e->host_turn + kTurns * (kReps + 1) > e->n_turns)
        return BLOND_OK;
    const size_t S = (size_t)e->S, n = (size_t)e->n, esz = energy_bytes(e->precision);
    char* snap = nullptr;
    if (cudaMalloc(&snap, 16 + 16 * S) != cudaSuccess) {
        cudaGetLastError();
        return BLOND_OK;  // no room for the snapshot: keep the setting
    }
    double* svind = reinterpret_cast<double*>(snap + 16);
    double* sprof = svind + S;
    cudaMemcpyAsync(snap, e->d_turn, sizeof(long long), cudaMemcpyDeviceToDevice, s);
    if (e->d_vind) cudaMemcpyAsync(svind, e->d_vind, 8 * S, cudaMemcpyDeviceToDevice, s);
    if (e->d_profile) cudaMemcpyAsync(sprof, e->d_profile, 8 * S, cudaMemcpyDeviceToDevice, s);
    auto restore = [&]() {
        cudaMemcpyAsync(e->dt, sdt, 8 * n, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(e->dE, sdE, esz * n, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(e->d_hist, shist, sizeof(int) * S, cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(e->d_turn, snap, sizeof(long long), cudaMemcpyDeviceToDevice, s);
        if (e->d_vind) cudaMemcpyAsync(e->d_vind, svind, 8 * S, cudaMemcpyDeviceToDevice, s);
        if (e->d_profile) cudaMemcpyAsync(e->d_profile, sprof, 8 * S, cudaMemcpyDeviceToDevice, s);
    };
    const bool keep = e->pdl;
    double t[2] = {0.0, 0.0};
    int rc = BLOND_OK;
    for (int on = 1; on >= 0 && rc == BLOND_OK; --on) {
        restore();
        e->pdl = on != 0;
        rc = time_graph_turns(e, s, kTurns, kReps, &t[on]);
    }
    restore();
    const cudaError_t ce = cudaStreamSynchronize(s);
    cudaFree(snap);
    if (rc == BLOND_OK && ce != cudaSuccess) {
        set_error("engine_autotune: %s", cudaGetErrorString(ce));
        rc = BLOND_ERR_CUDA;
    }
    // overlap stays on unless it is clearly slower
    e->pdl = rc == BLOND_OK ? !(t[0] < 0.97 * t[1]) : keep;
    *chosen = e->pdl ? 1 : 0;
    return rc;
}

}  // namespace bb

extern "C" {

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
    const size_t esz = energy_bytes(e->precision);
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
    struct Cand { int variant, threads, bps, hist, ring, cluster, l2 = 0; };
    std::vector<Cand> cands;
    std::vector<int> plain_modes;
    if (global_hist(e)) plain_modes = {HIST_GLOBAL};
    else if (e->S <= 2048) plain_modes = {HIST_AGG, HIST_I32, HIST_GLOBAL};
    else plain_modes = {HIST_I32, HIST_GLOBAL};
    // shared-memory sizes depend only on the stored energy's size, which is
    // 4 bytes in both F32P64 and Q32P64
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
    // the shared-table pass (packed histogram), with and without the ring
    for (int ring : {0, 2}) {
        const int sm = f64 ? stab_smem<PREC_F64>(e, ring) : stab_smem<PREC_F32P64>(e, ring);
        if (sm >= 0) cands.push_back({2, kEngineThreads, 1, HIST_PACKED, ring, 1, 0});
        if (sm >= 0 && ring) cands.push_back({2, kEngineThreads, 1, HIST_PACKED, ring, 1, 1});
    }
    // the plain pass with a packed histogram over the global table (long profiles)
    if (e->has_fft || e->has_ind || e->interp)
        for (int ring : {0, 2, 4}) {
            const int sm = f64 ? packed_smem<PREC_F64>(e, ring) : packed_smem<PREC_F32P64>(e, ring);
            if (sm >= 0) cands.push_back({3, kEngineThreads, 1, HIST_PACKED, ring, 1, 0});
        }
    const Cand old = {e->variant, e->threads, e->blocks_per_sm, e->hist_mode, e->ring,
                      e->cluster, e->l2_ahead ? 1 : 0};
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
        e->l2_ahead = c.l2 != 0;
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
    // whole turns with the winner: overlap on or off
    int overlap = e->pdl ? 1 : 0;
    if (rc == BLOND_OK && best < 1e30) {
        e->variant = win.variant;
        e->threads = win.threads;
        e->blocks_per_sm = win.bps;
        e->hist_mode = win.hist;
        e->ring = win.ring;
        e->cluster = win.cluster;
        e->l2_ahead = win.l2 != 0;
        rc = tune_overlap(e, s, sdt, sdE, static_cast<const int*>(shist), &overlap);
    }
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
    e->l2_ahead = use.l2 != 0;
    e->graph_dirty = true;
    config[0] = use.variant;
    config[1] = use.variant == 1 ? use.threads : (use.variant == 0 ? kTmaThreads : kEngineThreads);
    // (variants 2 and 3 run 1024 threads x one block per SM)
    config[2] = use.variant == 1 ? use.bps : 1;
    config[3] = use.hist;
    config[4] = use.ring;
    config[5] = use.cluster;
    config[6] = use.l2;
    config[7] = (int)cands.size();
    config[8] = overlap;
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
    if (e->smooth) {
        set_error("engine_track_host: smooth slicing reads the whole beam after the pass; "
                  "track device-resident coordinates");
        return BLOND_ERR_UNSUPPORTED;
    }
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
    const size_t esz = energy_bytes(e->precision);
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
    if (e->smooth) {
        set_error("engine_set_feedback: not with smooth slicing");
        return BLOND_ERR_UNSUPPORTED;
    }
    if (e->interp && (machine == BLOND_FB_SPS_RL || !e->has_fft)) {
        set_error("engine_set_feedback: an interpolated turn takes no SPS_RL loop, and other "
                  "loops only with an FFT impedance");
        return BLOND_ERR_UNSUPPORTED;
    }
    if (machine == BLOND_FB_SPS_RL && e->precision == BLOND_PREC_Q32P64) {
        set_error("engine_set_feedback: the SPS_RL loop's energy average is not built for "
                  "fixed-point energies (Q32P64)");
        return BLOND_ERR_UNSUPPORTED;
    }
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

// Largest profile the fixed scratch holds.  Profiles this short keep their
// histogram in shared memory, so the entry point always runs the plain
// particle pass, which has no bounded waits: the scratch error word below
// is never set by it (checked at run time before the launch).
constexpr int kNoAllocMaxSlices = 16384;

struct NoAllocScratch {
    int hist[kNoAllocMaxSlices];              // integer slice counts
    double2 table[kNoAllocMaxSlices];         // interpolation table
    double bc[kNoAllocMaxSlices];             // bin centres
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

// This call's constants, passed to the set-up kernel by value.
struct NoAllocHead {
    DriftTurn drift;
    double acc;
    double cut_left, cut_right;
    int S;
};

// Per-call set-up on the stream: the histogram starts at zero (the
// previous call leaves its last counts behind), the bin centres, this
// turn's drift constants and kick, the turn counter and the error word.
__global__ void noalloc_setup_kernel(NoAllocScratch* sc, const NoAllocHead h) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < h.S; k += gridDim.x * blockDim.x) {
        sc->hist[k] = 0;
        sc->bc[k] = linspace_centre(h.cut_left, h.cut_right, h.S, k);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sc->drift[0] = h.drift;
        sc->drift[1] = h.drift;
        sc->acc = h.acc;
        sc->turn = 0;
        sc->err = 0;
    }
}

}  // namespace bb

extern "C" int blond_turn_f64_noalloc(
    double* dt, double* dE, int64_t n, int n_rf, double charge, const double* voltage,
    const double* omega_rf, const double* phi_rf, double acc_kick, int solver,
    double t_rev, double length_ratio, double alpha_order, double eta_0, double eta_1,
    double eta_2, double alpha_0, double alpha_1, double alpha_2, double beta,
    double energy, double cut_left, double cut_right, int n_slices,
    const double* impedance, int64_t n_fft, double iv_scale, double* profile_out,
    double* induced_voltage_out, void* stream) {
    using namespace bb;
    BB_CHECK_ARG(dt && dE && voltage && omega_rf && phi_rf && profile_out,
                 "turn_noalloc: null pointer");
    BB_CHECK_ARG(n >= 1, "turn_noalloc: n must be >= 1");
    BB_CHECK_ARG(solver >= 0 && solver <= 2, "turn_noalloc: solver %d", solver);
    BB_CHECK_ARG(aligned(dt, 16) && aligned(dE, 16),
                 "turn_noalloc: dt and dE must be 16-byte aligned");
    BB_CHECK_ARG(std::isfinite(cut_left) && std::isfinite(cut_right) && cut_right > cut_left,
                 "turn_noalloc: need finite cuts with cut_right > cut_left");
    BB_CHECK_ARG(beta > 0 && energy > 0, "turn_noalloc: beta and energy must be > 0");
    BB_CHECK_SIZE(n_rf >= 1 && n_rf <= kMaxRfEngine, "turn_noalloc: n_rf=%d not in [1, %d]",
                  n_rf, kMaxRfEngine);
    BB_CHECK_SIZE(n_slices >= 2 && n_slices <= kNoAllocMaxSlices,
                  "turn_noalloc: n_slices=%d exceeds the fixed scratch (2..%d slices); "
                  "use the engine API for longer profiles", n_slices, kNoAllocMaxSlices);
    const double bc0 = linspace_centre(cut_left, cut_right, n_slices, 0);
    const double bc1 = linspace_centre(cut_left, cut_right, n_slices, 1);
    const double bcl = linspace_centre(cut_left, cut_right, n_slices, n_slices - 1);
    BB_CHECK_ARG(bcl > bc0 && bc1 > bc0, "turn_noalloc: the slicing window is too narrow "
                 "for %d distinct bin centres", n_slices);
    SpecPlan plan = {};
    if (impedance) {
        BB_CHECK_ARG(induced_voltage_out, "turn_noalloc: null induced_voltage_out");
        BB_CHECK_ARG(aligned(impedance, 16),
                     "turn_noalloc: impedance must be 16-byte aligned (complex128)");
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
    // engine does per turn), handed to the set-up kernel by value
    NoAllocHead h = {};
    DriftTurn& d = h.drift;
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
    h.acc = acc_kick;
    h.cut_left = cut_left;
    h.cut_right = cut_right;
    h.S = n_slices;
    noalloc_setup_kernel<<<std::min(64, (n_slices + 255) / 256), 256, 0, s>>>(sc, h);
    BB_LAUNCH_CHECK();

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
    e.bc0 = bc0;
    e.lik_inv_w = (n_slices - 1) / (bcl - bc0);
    e.bw = 1.0 / e.lik_inv_w;
    e.dbc = bc1 - bc0;
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
    // the plain pass (no bounded waits, so no error word to report) needs
    // the histogram in shared memory
    if (global_hist(&e)) {
        set_error("turn_noalloc: %d slices do not fit a shared-memory histogram here",
                  n_slices);
        return BLOND_ERR_UNSUPPORTED;
    }

    int rc;
    if ((rc = launch_particles(&e, false, s))) return rc;  // slice the input
    if ((rc = launch_head(&e, s))) return rc;              // profile, V, table
    if ((rc = launch_particles(&e, true, s))) return rc;   // the turn
    return launch_profile(&e, false, s);                   // final profile
}

