// Batched engine: many independent beams tracked by one particle launch
// and one head launch per turn.
#include "engine_device.cuh"

// ============================================================ batched beams
// Many independent beams (ragged particle counts, own RF programme, slicing
// window and impedance each) tracked together: ONE particle launch and ONE
// head launch per turn for the whole batch.  Particles are concatenated;
// a chunk table cuts every beam into pieces of at most `chunk` particles,
// each piece processed by one block with its beam's constants in shared
// memory and a private shared-memory histogram flushed to the beam's
// global histogram.  The head kernel runs one cluster per beam.  Each beam
// follows exactly the arithmetic of the single-beam engine (track_pair).
//
// Launch shape (blond_batch_autotune picks it, blond_batch_set_shape fixes
// it): threads per block, blocks per SM, particles per thread and
// iteration (2, 4 or 8, all loads issued before any arithmetic), chunk
// size, and plain or warp-aggregated shared-memory deposits.
namespace bb {

constexpr int kBatchChunkDefault = 32768;
constexpr int kBatchMaxThreads = 1024;
// Largest histogram + table copy per block (four 256-thread blocks per SM
// stay resident).
constexpr size_t kBatchTableSmem = 48 * 1024;

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
    int B;
    const double* cut_left;     // [B]
    const double* inv_w;        // [B]
    const double* bc0;          // [B]
    const double* lik_inv_w;    // [B]
    const double* bw;           // [B]
    int* hist;                  // [B][S]
    const void* table;          // [B][S]
    const double* lsb;          // Q32P64: [2B] energy unit per beam, then its inverse
    int* err;                   // sticky error word (ERR_ENERGY_RANGE)
    int agg;                    // warp-aggregated shared-memory deposits
    unsigned* next_chunk;       // chunks claimed beyond the first wave (zero between launches)
};

// Block b starts on chunk b; afterwards each block claims the next unclaimed
// chunk (chunks are sorted by size, largest first, so the launch ends on
// small ones and the blocks finish together).  There are n_chunks claims
// per launch (every chunk past the first wave once, plus one failed claim
// per block); the block making the last one resets the counter for the
// next launch, when no block of this launch touches it any more.
__device__ __forceinline__ int claim_chunk(unsigned* counter, int n_chunks) {
    const unsigned v = atomicAdd(counter, 1u);
    if (v == (unsigned)n_chunks - 1u) *counter = 0u;
    return (int)gridDim.x + (int)v;
}

// The launch bound (1024 threads, one block) caps registers at 64 a thread,
// so every shape with at most 1024 resident threads per SM runs the same
// code.
// TSM: the beam's interpolation table is copied into shared memory (after
// the histogram) at the start of every chunk, for short profiles.
template <int PREC, int SOLVER, bool LIK, bool KICK, int PPT, bool TSM = false>
__global__ void __launch_bounds__(kBatchMaxThreads, 1)
particle_kernel_batch(const BatchArgs a) {
    using E = typename Coord<PREC>::E;
    using TB = typename TableEntry<PREC>::T;
    static_assert(PPT == 2 || PPT == 4 || PPT == 8, "particles per thread");
    extern __shared__ __align__(16) int sh[];
    TB* stab = reinterpret_cast<TB*>(reinterpret_cast<char*>(sh) + pad16((size_t)a.S * 4));
    __shared__ TurnConsts c;
    long long t = a.turn ? (*a.turn - 1) : 0;
    if (t < 0) t = 0;
    if (t >= a.n_turns) t = a.n_turns - 1;
    double* dt = reinterpret_cast<double*>(a.dt);
    E* dE = reinterpret_cast<E*>(a.dE);
    const int S = a.S;
    const uint64_t pol = evict_first_policy();
    __shared__ int next;
    for (int ch = blockIdx.x; ch < a.n_chunks; ch = next) {
        const int b = a.chunk_beam[ch];
        const long long start = a.chunk_start[ch];
        const int count = a.chunk_count[ch];
        if (KICK) {
            const long long rb = (long long)b * (a.n_turns + 1);
            for (int j = threadIdx.x; j < a.n_rf; j += blockDim.x) {
                c.V[j] = a.V[(rb + t) * a.n_rf + j];
                c.Vf[j] = (float)c.V[j];
                c.op[j] = make_double2(a.om[(rb + t) * a.n_rf + j], a.ph[(rb + t) * a.n_rf + j]);
            }
            if (threadIdx.x == 0) {
                c.acc = a.acc[(long long)b * a.n_turns + t];
                c.d = a.drift[rb + t + 1];
            }
        }
        if constexpr (TSM && LIK) {
            // the beam's S - 1 entries (L2-resident), asynchronously, one
            // entry-sized copy each (entries are 16- or 8-byte aligned)
            const TB* src = reinterpret_cast<const TB*>(a.table) + (long long)b * S;
            for (int k = threadIdx.x; k < S - 1; k += blockDim.x) {
                if constexpr (sizeof(TB) == 16) copy16_async(&stab[k], &src[k]);
                else copy8_async(&stab[k], &src[k]);
            }
            ring_commit();
        }
        for (int k = threadIdx.x; k < S; k += blockDim.x) sh[k] = 0;
        if constexpr (TSM && LIK) ring_wait<0>();
        __syncthreads();
        ParticleArgs pa = {};
        pa.n_rf = a.n_rf;
        pa.charge = a.charge;
        pa.S = S;
        pa.bc0 = a.bc0[b];
        pa.lik_inv_w = a.lik_inv_w[b];
        pa.bw = a.bw[b];
        pa.table = LIK ? static_cast<const char*>(a.table) +
                             (long long)b * S * sizeof(typename TableEntry<PREC>::T)
                       : nullptr;
        if (PREC == PREC_Q32P64) {
            pa.lsb = a.lsb[b];
            pa.inv_lsb = a.lsb[a.B + b];
        }
        pa.err = a.err;
        const double cl = a.cut_left[b], iw = a.inv_w[b];
        // PPT particles per thread and iteration (i + q * blockDim), all
        // loads issued before any arithmetic (two per thread left ~16 KB of
        // loads in flight per SM, which capped HBM near 2.4 TB/s).  Whole
        // warps iterate together, so the aggregated deposit's warp vote
        // sees every lane.
        // PPT particles per thread and iteration as PPT / 2 pairs of
        // neighbours (one 16-byte dt load, one pair-sized dE load each), all
        // loads issued before any arithmetic (two particles per thread left
        // ~16 KB of loads in flight per SM, which capped HBM near 2.4 TB/s).
        // Pairs start on an even particle index; an odd first particle and
        // an unpaired last one go through the same arithmetic below.  Whole
        // warps iterate together, so the aggregated deposit's warp vote sees
        // every lane.
        using E2 = typename Vec2<E>::type;
        constexpr int PP = PPT / 2;
        const int bd = blockDim.x;
        const int lane_base = threadIdx.x & ~31;
        const int head = (int)(start & 1);
        const long long p0 = (start + head) >> 1;  // first pair
        const int npair = (count - head) >> 1;
        const double2* dt2 = reinterpret_cast<const double2*>(dt);
        const E2* dE2 = reinterpret_cast<const E2*>(dE);
        for (int w = lane_base; w < npair; w += PP * bd) {
            const int j = w + (threadIdx.x & 31);
            // F32P64: thread 0 prefetches the block's next iteration into L2
            // (C3: 2.059 -> 2.040 ms per turn)
            if (PREC == PREC_F32P64 && threadIdx.x == 0 && w + PP * bd < npair) {
                const long long lo = 2 * (p0 + w + (long long)PP * bd);
                const long long hi = 2 * (p0 + min((long long)npair, (long long)w + 2LL * PP * bd));
                l2_prefetch_range(dt + lo, dt + hi, pol);
                l2_prefetch_range(dE + lo, dE + hi, pol);
            }
            double2 tq[PP];
            E2 e[PP];
            bool in[PP];
#pragma unroll
            for (int q = 0; q < PP; ++q) {
                in[q] = j + q * bd < npair;
                const long long g = p0 + (in[q] ? j + q * bd : 0);
                tq[q] = stream_load(dt2 + g, pol);
                e[q] = stream_load(dE2 + g, pol);
            }
            if (KICK) {
#pragma unroll
                for (int q = 0; q < PP; ++q)
                    track_pair<PREC, SOLVER, LIK, (TSM && LIK) ? TAB_ENTRIES : TAB_GLOBAL, true>(
                        tq[q].x, tq[q].y, e[q].x, e[q].y, c, pa, a.order, stab);
#pragma unroll
                for (int q = 0; q < PP; ++q) {
                    if (in[q]) {
                        stream_store(reinterpret_cast<double2*>(dt) + p0 + j + q * bd, tq[q], pol);
                        stream_store(reinterpret_cast<E2*>(dE) + p0 + j + q * bd, e[q], pol);
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < PP; ++q) {
                const int b0 = in[q] ? engine_bin(tq[q].x, cl, iw, S) : -1;
                const int b1 = in[q] ? engine_bin(tq[q].y, cl, iw, S) : -1;
                if (a.agg) {
                    deposit(sh, b0, true, 0xffffffffu);
                    deposit(sh, b1, true, 0xffffffffu);
                } else {
                    if (b0 >= 0) atomicAdd(&sh[b0], 1);
                    if (b1 >= 0) atomicAdd(&sh[b1], 1);
                }
            }
        }
        // the odd first particle (thread 0) and the unpaired last one (thread 1)
        if (threadIdx.x < 2 && (threadIdx.x == 0 ? head : (count - head) & 1)) {
            const long long g = threadIdx.x == 0 ? start : start + count - 1;
            double t0 = dt[g], t1 = t0;
            E e0 = dE[g], e1 = e0;
            if (KICK) {
                track_pair<PREC, SOLVER, LIK, (TSM && LIK) ? TAB_ENTRIES : TAB_GLOBAL, true>(
                    t0, t1, e0, e1, c, pa, a.order, stab);
                dt[g] = t0;
                dE[g] = e0;
            }
            const int bq = engine_bin(t0, cl, iw, S);
            if (bq >= 0) atomicAdd(&sh[bq], 1);
        }
        __syncthreads();
        for (int k = threadIdx.x; k < S; k += blockDim.x) {
            const int v = sh[k];
            if (v) atomicAdd(&a.hist[(long long)b * S + k], v);
        }
        if (threadIdx.x == 0) next = claim_chunk(a.next_chunk, a.n_chunks);
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
    std::vector<int64_t> offsets;  // host copy of the beams' offsets (B + 1)
    double* d_lsb = nullptr;       // Q32P64: [2B] energy units, then inverses
    bool lsb_set = false;
    int* d_err = nullptr;          // sticky error word of the particle pass
    unsigned* d_next_chunk = nullptr;  // the particle pass's chunk claims
    bool rf_set = false, drift_set = false, slicing_set = false;
    // launch shape of the particle pass
    int threads = 512, blocks_per_sm = 2, ppt = 4, chunk = bb::kBatchChunkDefault, agg = 0;
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
    a.B = q->B;
    a.lsb = q->d_lsb;
    a.err = q->d_err;
    a.agg = q->agg;
    a.next_chunk = q->d_next_chunk;
    return a;
}

// Shared memory of the batched pass: the histogram, and with the table
// copy (short profiles) the table after it; 0 when the copy does not fit.
template <int PREC>
static int batch_table_smem(const blond_batch* q) {
    const size_t bytes = pad16((size_t)q->S * 4) +
                         pad16((size_t)(q->S - 1) * sizeof(typename TableEntry<PREC>::T));
    return bytes <= kBatchTableSmem ? (int)bytes : 0;
}

template <int PREC, int SOLVER, bool LIK, bool KICK, int PPT>
static int launch_batch_k(blond_batch* q, cudaStream_t s, bool launch) {
    static bool done[64] = {false};
    static bool done_t[64] = {false};
    const int tsm = (LIK && KICK) ? batch_table_smem<PREC>(q) : 0;
    auto k = tsm ? particle_kernel_batch<PREC, SOLVER, LIK, KICK, PPT, true>
                 : particle_kernel_batch<PREC, SOLVER, LIK, KICK, PPT, false>;
    int rc;
    if ((rc = allow_max_smem(k, tsm ? done_t : done))) return rc;
    if (!launch) return BLOND_OK;
    const int smem = tsm ? tsm : (int)sizeof(int) * q->S;
    const int grid = std::max(1, std::min(q->n_chunks, device_info().sm_count * q->blocks_per_sm));
    k<<<grid, q->threads, smem, s>>>(batch_args(q));
    BB_LAUNCH_CHECK();
    return BLOND_OK;
}

template <int PREC, int SOLVER, bool LIK, bool KICK>
static int launch_batch_t(blond_batch* q, cudaStream_t s, bool launch) {
    if (!KICK) return launch_batch_k<PREC, SOLVER, LIK, KICK, 4>(q, s, launch);
    switch (q->ppt) {
        case 2: return launch_batch_k<PREC, SOLVER, LIK, KICK, 2>(q, s, launch);
        case 8: return launch_batch_k<PREC, SOLVER, LIK, KICK, 8>(q, s, launch);
        default: return launch_batch_k<PREC, SOLVER, LIK, KICK, 4>(q, s, launch);
    }
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
    switch (q->precision) {
        case BLOND_PREC_F64: return launch_batch_p<PREC_F64>(q, kick, s, launch);
        case BLOND_PREC_F32P64: return launch_batch_p<PREC_F32P64>(q, kick, s, launch);
        default: return launch_batch_p<PREC_Q32P64>(q, kick, s, launch);
    }
}

// Cut every beam into chunks of at most q->chunk particles (one block's
// piece of work), largest first (the blocks claim them in this order), and
// upload the chunk table.
static int batch_rechunk(blond_batch* q) {
    struct Chunk { long long start; int beam, count; };
    std::vector<Chunk> all;
    for (int b = 0; b < q->B; ++b) {
        for (int64_t s0 = q->offsets[b]; s0 < q->offsets[b + 1]; s0 += q->chunk)
            all.push_back({s0, b, (int)std::min<int64_t>(q->chunk, q->offsets[b + 1] - s0)});
    }
    std::stable_sort(all.begin(), all.end(),
                     [](const Chunk& x, const Chunk& y) { return x.count > y.count; });
    std::vector<long long> cs;
    std::vector<int> cb, cc;
    for (const Chunk& c : all) {
        cs.push_back(c.start);
        cb.push_back(c.beam);
        cc.push_back(c.count);
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
    q->graph_dirty = true;
    return BLOND_OK;
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
    if (q->precision == BLOND_PREC_Q32P64 && !q->lsb_set) {
        set_error("batch: precision Q32P64 needs set_energy_units before tracking");
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
    BB_CHECK_ARG(precision == BLOND_PREC_F64 || precision == BLOND_PREC_F32P64 ||
                     precision == BLOND_PREC_Q32P64,
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
        cudaMalloc(&q->d_err, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&q->d_next_chunk, sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&q->d_hist, sizeof(int) * bs) != cudaSuccess ||
        cudaMalloc(&q->d_profile, sizeof(double) * bs) != cudaSuccess ||
        cudaMalloc(&q->d_vind, sizeof(double) * bs) != cudaSuccess ||
        cudaMalloc(&q->d_table, sizeof(double2) * bs) != cudaSuccess ||
        cudaStreamCreateWithFlags(&q->cap_stream, cudaStreamNonBlocking) != cudaSuccess) {
        set_error("batch_create: allocation failed");
        rc = BLOND_ERR_CUDA;
    } else {
        cudaMemset(q->d_turn, 0, sizeof(long long));
        cudaMemset(q->d_err, 0, sizeof(int));
        cudaMemset(q->d_next_chunk, 0, sizeof(unsigned));
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
                    (void*)q->d_profile, (void*)q->d_vind, q->d_table, (void*)q->d_turn,
                    (void*)q->d_lsb, (void*)q->d_err, (void*)q->d_next_chunk})
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
    // With at least one beam per two SMs, one CTA per beam when the whole
    // transform fits in its shared memory: no cluster barriers, and the
    // beams themselves fill the GPU
    SpecPlan one;
    if (q->B * 2 >= device_info().sm_count && make_spec_plan(n_fft, one, 1) &&
        one.smem <= device_info().max_smem_optin)
        plan = one;
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
    BB_CHECK_ARG(aligned(dt, 16) && aligned(dE, 16),
                 "batch_bind_beams: dt and dE must be 16-byte aligned");
    BB_CHECK_ARG(offsets[0] == 0, "batch_bind_beams: offsets[0] must be 0");
    for (int b = 0; b < q->B; ++b)
        BB_CHECK_ARG(offsets[b + 1] >= offsets[b], "batch_bind_beams: offsets decrease");
    q->offsets.assign(offsets, offsets + q->B + 1);
    int rc = batch_rechunk(q);
    if (rc) return rc;
    q->dt = dt;
    q->dE = dE;
    q->n_total = offsets[q->B];
    q->graph_dirty = true;
    return BLOND_OK;
}

int blond_batch_set_energy_units(blond_batch* q, const double* lsb) {
    using namespace bb;
    BB_CHECK_ARG(q && lsb, "batch_set_energy_units: null pointer");
    std::vector<double> u(2 * (size_t)q->B);
    for (int b = 0; b < q->B; ++b) {
        BB_CHECK_ARG(std::isfinite(lsb[b]) && lsb[b] > 0, "batch_set_energy_units: beam %d: "
                     "the unit must be a finite energy > 0 (eV per count)", b);
        u[b] = lsb[b];
        u[q->B + b] = 1.0 / lsb[b];
    }
    int rc = upload((void**)&q->d_lsb, u.data(), sizeof(double) * u.size());
    if (rc) return rc;
    q->lsb_set = true;
    q->graph_dirty = true;
    return BLOND_OK;
}

int blond_batch_check(blond_batch* q, void* stream) {
    using namespace bb;
    BB_CHECK_ARG(q, "batch_check: null batch");
    int flag = 0;
    BB_CUDA(cudaMemcpyAsync(&flag, q->d_err, sizeof(int), cudaMemcpyDeviceToHost,
                            as_stream(stream)));
    BB_CUDA(cudaStreamSynchronize(as_stream(stream)));
    if (flag) {
        BB_CUDA(cudaMemsetAsync(q->d_err, 0, sizeof(int), as_stream(stream)));
        set_error("batch: an energy left the 32-bit fixed-point grid of its beam; track "
                  "again with a larger energy unit");
        return BLOND_ERR_RANGE;
    }
    return BLOND_OK;
}

int blond_batch_set_shape(blond_batch* q, int threads, int blocks_per_sm,
                          int particles_per_thread, int chunk, int aggregate) {
    using namespace bb;
    BB_CHECK_ARG(q, "batch_set_shape: null batch");
    BB_CHECK_ARG(threads % 32 == 0 && threads >= 64 && threads <= kBatchMaxThreads,
                 "batch_set_shape: threads must be a multiple of 32 in [64, %d]",
                 kBatchMaxThreads);
    BB_CHECK_ARG(blocks_per_sm >= 1 && threads * blocks_per_sm <= 2048,
                 "batch_set_shape: blocks_per_sm must be >= 1 with <= 2048 threads per SM");
    BB_CHECK_ARG(particles_per_thread == 2 || particles_per_thread == 4 ||
                     particles_per_thread == 8,
                 "batch_set_shape: particles_per_thread must be 2, 4 or 8");
    BB_CHECK_ARG(chunk >= 1024 && chunk <= (1 << 22),
                 "batch_set_shape: chunk must be in [1024, 2^22]");
    q->threads = threads;
    q->blocks_per_sm = blocks_per_sm;
    q->ppt = particles_per_thread;
    q->agg = aggregate ? 1 : 0;
    if (chunk != q->chunk) {
        q->chunk = chunk;
        if (!q->offsets.empty()) {
            int rc = batch_rechunk(q);
            if (rc) return rc;
        }
    }
    q->graph_dirty = true;
    return BLOND_OK;
}

// Time every launch shape of the particle pass on the bound beams (CUDA
// events, one warm-up + reps launches each, the coordinates and histograms
// restored afterwards) and keep the fastest.  config receives {threads,
// blocks_per_sm, particles_per_thread, chunk, aggregate, candidates}.
int blond_batch_autotune(blond_batch* q, int reps, void* stream, int* config,
                         double* best_ms) {
    using namespace bb;
    BB_CHECK_ARG(q && config && best_ms && reps >= 1 && reps <= 10,
                 "batch_autotune: bad argument (reps in 1..10)");
    int rc = batch_ready(q);
    if (rc) return rc;
    cudaStream_t s = as_stream(stream);
    cudaStreamCaptureStatus cs;
    BB_CUDA(cudaStreamIsCapturing(s, &cs));
    BB_CHECK_ARG(cs == cudaStreamCaptureStatusNone, "batch_autotune: the stream is being captured");
    const size_t esz = q->precision == BLOND_PREC_F64 ? sizeof(double) : 4;
    const size_t n = (size_t)q->n_total, hs = sizeof(int) * (size_t)q->B * q->S;
    void *sdt = nullptr, *sdE = nullptr, *shist = nullptr;
    if (cudaMalloc(&sdt, 8 * n + 8) != cudaSuccess || cudaMalloc(&sdE, esz * n + 8) != cudaSuccess ||
        cudaMalloc(&shist, hs) != cudaSuccess) {
        free_ptr(sdt);
        free_ptr(sdE);
        free_ptr(shist);
        cudaGetLastError();
        set_error("batch_autotune: cannot allocate the snapshot (%zu bytes)", (8 + esz) * n);
        return BLOND_ERR_CUDA;
    }
    BB_CUDA(cudaMemcpyAsync(sdt, q->dt, 8 * n, cudaMemcpyDeviceToDevice, s));
    BB_CUDA(cudaMemcpyAsync(sdE, q->dE, esz * n, cudaMemcpyDeviceToDevice, s));
    BB_CUDA(cudaMemcpyAsync(shist, q->d_hist, hs, cudaMemcpyDeviceToDevice, s));
    struct Cand { int threads, bps, ppt, chunk, agg; };
    const Cand old = {q->threads, q->blocks_per_sm, q->ppt, q->chunk, q->agg};
    std::vector<Cand> cands;
    for (int chunk : {16384, 32768, 65536})
        for (int threads : {256, 512, 1024})
            for (int bps : {1, 2, 4})
                // 64 registers a thread: at most 1024 threads resident per SM
                if (threads * bps <= 1024)
                    for (int ppt : {2, 4, 8})
                        for (int agg : {0, 1}) cands.push_back({threads, bps, ppt, chunk, agg});
    cudaEvent_t a = nullptr, b = nullptr;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    double best = 1e30;
    Cand win = old;
    for (const Cand& c : cands) {
        if ((rc = blond_batch_set_shape(q, c.threads, c.bps, c.ppt, c.chunk, c.agg))) break;
        if ((rc = launch_batch(q, true, s, false))) break;
        if ((rc = launch_batch(q, true, s))) break;  // warm-up
        cudaEventRecord(a, s);
        for (int r = 0; r < reps && rc == BLOND_OK; ++r) rc = launch_batch(q, true, s);
        cudaEventRecord(b, s);
        if (rc) break;
        if (cudaEventSynchronize(b) != cudaSuccess) {
            set_error("batch_autotune: a candidate failed");
            rc = BLOND_ERR_CUDA;
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (ms / reps < best) {
            best = ms / reps;
            win = c;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    // restore the state of the run
    cudaMemcpyAsync(q->dt, sdt, 8 * n, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(q->dE, sdE, esz * n, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(q->d_hist, shist, hs, cudaMemcpyDeviceToDevice, s);
    const cudaError_t ce = cudaStreamSynchronize(s);
    free_ptr(sdt);
    free_ptr(sdE);
    free_ptr(shist);
    if (rc == BLOND_OK && ce != cudaSuccess) {
        set_error("batch_autotune: %s", cudaGetErrorString(ce));
        rc = BLOND_ERR_CUDA;
    }
    if (rc == BLOND_OK) rc = blond_batch_check(q, stream);
    const Cand& use = rc == BLOND_OK && best < 1e30 ? win : old;
    const int rc2 = blond_batch_set_shape(q, use.threads, use.bps, use.ppt, use.chunk, use.agg);
    if (rc == BLOND_OK) rc = rc2;
    config[0] = use.threads;
    config[1] = use.bps;
    config[2] = use.ppt;
    config[3] = use.chunk;
    config[4] = use.agg;
    config[5] = (int)cands.size();
    *best_ms = best < 1e30 ? best : 0.0;
    return rc;
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
