/*
 * blond_b200 -- C ABI of the B200 longitudinal tracking engine.
 *
 * All array arguments are DEVICE pointers (CUDA global memory on the current
 * device) unless a comment says "host".  Every call is asynchronous on the
 * given stream (a cudaStream_t passed as void*, NULL = legacy default
 * stream) and returns a status code; blond_b200_last_error() gives the
 * message of the last failure on the calling thread.  Lengths are int64_t.
 * Nothing here allocates memory visible to the caller; callers own every
 * array they pass.
 *
 * The bmath-level entry points mirror the reference's libblond exports
 * (the .cpp files of blond/cpp_routines, bound by blond/utils/butils_wrap_cpp.py) with
 * the same argument order and meaning; _f64 corresponds to
 * libblond_double.so and _f32 to libblond_single.so (blond_common.h:22-36).
 */
#ifndef BLOND_B200_H
#define BLOND_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ status codes */
#define BLOND_OK 0
#define BLOND_ERR_INVALID_ARGUMENT 1 /* null pointer, negative length, bad enum */
#define BLOND_ERR_SIZE 2             /* n_slices / n_fft / n_rf outside the supported range */
#define BLOND_ERR_ALIGNMENT 3        /* pointer not aligned to its element size */
#define BLOND_ERR_CUDA 4             /* CUDA runtime error (launch, allocation, graph) */
#define BLOND_ERR_UNSUPPORTED 5      /* e.g. an FFT length with a prime factor > 5 */
#define BLOND_ERR_TIMEOUT 6          /* a bounded device-side wait gave up */
#define BLOND_ERR_STATE 7            /* engine used before it was configured */
#define BLOND_ERR_RANGE 8            /* a fixed-point energy left its 32-bit grid */

/* drift solvers, as butils_wrap_cpp.drift maps them (butils_wrap_cpp.py:920-925) */
#define BLOND_SOLVER_SIMPLE 0
#define BLOND_SOLVER_LEGACY 1
#define BLOND_SOLVER_EXACT 2

/* fused-engine precision modes */
#define BLOND_PREC_F64 0    /* dt, dE float64; all arithmetic float64 (plain) */
#define BLOND_PREC_F32P64 1 /* dt float64, dE float32; RF phase argument and
                               drift in float64, kick arithmetic in float32 */
#define BLOND_PREC_Q32P64 2 /* dt float64, dE int32 counts of a per-beam energy
                               unit (set_energy_unit); kick and drift
                               arithmetic in float64, the energy rounded to
                               the unit once per turn */

const char* blond_b200_last_error(void);
int blond_b200_version(void);
/* Largest n_slices the shared-memory histogram privatises (bins beyond it
 * fall back to global atomics); informational. */
int blond_b200_max_smem_slices(void);

/* ------------------------------------------------------------ RF kick
 * replaces kick()          cpp_routines/kick.cpp:16-35
 *   dE[i] += charge * sum_j voltage[j] sin(omega_rf[j] dt[i] + phi_rf[j]) + acc_kick
 * voltage/omega_rf/phi_rf: n_rf device values (one turn column). */
int blond_kick_f64(const double* dt, double* dE, int n_rf, double charge,
                   const double* voltage, const double* omega_rf,
                   const double* phi_rf, int64_t n, double acc_kick,
                   void* stream);
int blond_kick_f32(const float* dt, float* dE, int n_rf, float charge,
                   const float* voltage, const float* omega_rf,
                   const float* phi_rf, int64_t n, float acc_kick,
                   void* stream);

/* replaces rf_volt_comp()  cpp_routines/kick.cpp:37-51  (accumulates: +=) */
int blond_rf_volt_comp_f64(const double* voltage, const double* omega_rf,
                           const double* phi_rf, const double* bin_centers,
                           int n_rf, int64_t n_bins, double* rf_voltage,
                           void* stream);
int blond_rf_volt_comp_f32(const float* voltage, const float* omega_rf,
                           const float* phi_rf, const float* bin_centers,
                           int n_rf, int64_t n_bins, float* rf_voltage,
                           void* stream);

/* ------------------------------------------------------------ drift
 * replaces drift()         cpp_routines/drift.cpp:19-78 (solver 0/1/2) */
int blond_drift_f64(double* dt, const double* dE, int solver, double t_rev,
                    double length_ratio, double alpha_order, double eta_0,
                    double eta_1, double eta_2, double alpha_0,
                    double alpha_1, double alpha_2, double beta,
                    double energy, int64_t n, void* stream);
int blond_drift_f32(float* dt, const float* dE, int solver, float t_rev,
                    float length_ratio, float alpha_order, float eta_0,
                    float eta_1, float eta_2, float alpha_0, float alpha_1,
                    float alpha_2, float beta, float energy, int64_t n,
                    void* stream);

/* ------------------------------------------------------------ slicing
 * replaces histogram()        cpp_routines/histogram.cpp:22-73
 * profile[n_slices] is OVERWRITTEN with the counts (exact integers). */
int blond_histogram_f64(const double* dt, double* profile, double cut_left,
                        double cut_right, int n_slices, int64_t n,
                        void* stream);
int blond_histogram_f32(const float* dt, float* profile, float cut_left,
                        float cut_right, int n_slices, int64_t n,
                        void* stream);
/* replaces smooth_histogram() cpp_routines/histogram.cpp:75-132 (overwrites) */
int blond_smooth_histogram_f64(const double* dt, double* profile,
                               double cut_left, double cut_right,
                               int n_slices, int64_t n, void* stream);
int blond_smooth_histogram_f32(const float* dt, float* profile,
                               float cut_left, float cut_right, int n_slices,
                               int64_t n, void* stream);

/* ------------------------------------------------------------ interpolated kick
 * replaces linear_interp_kick() cpp_routines/linear_interp_kick.cpp:21-71 */
int blond_linear_interp_kick_f64(const double* dt, double* dE,
                                 const double* voltage,
                                 const double* bin_centers, double charge,
                                 int n_slices, int64_t n, double acc_kick,
                                 void* stream);
int blond_linear_interp_kick_f32(const float* dt, float* dE,
                                 const float* voltage,
                                 const float* bin_centers, float charge,
                                 int n_slices, int64_t n, float acc_kick,
                                 void* stream);

/* ------------------------------------------------------------ beam phase
 * replaces beam_phase() and beam_phase_fast() cpp_routines/beam_phase.cpp:6-65
 * (bound at butils_wrap_cpp.py:785-832, called by BeamFeedback.beam_phase,
 * llrf/beam_feedback.py:276-309):
 *   coeff = T[w p sin(omega_rf bc + phi_rf)] / T[w p cos(omega_rf bc + phi_rf)]
 * with w = exp(alpha bc) (beam_phase) or 1 (beam_phase_fast) and T the
 * constant-step trapezoid of blondmath.cpp:496-512.  The reference returns
 * the value; here it is written to coeff, ONE device value, on the stream. */
int blond_beam_phase_f64(const double* bin_centers, const double* profile,
                         double alpha, double omega_rf, double phi_rf,
                         double bin_size, int n_bins, double* coeff,
                         void* stream);
int blond_beam_phase_f32(const float* bin_centers, const float* profile,
                         float alpha, float omega_rf, float phi_rf,
                         float bin_size, int n_bins, float* coeff,
                         void* stream);
int blond_beam_phase_fast_f64(const double* bin_centers, const double* profile,
                              double omega_rf, double phi_rf, double bin_size,
                              int n_bins, double* coeff, void* stream);
int blond_beam_phase_fast_f32(const float* bin_centers, const float* profile,
                              float omega_rf, float phi_rf, float bin_size,
                              int n_bins, float* coeff, void* stream);

/* ------------------------------------------------------------ beam statistics
 * replaces Beam.statistics() beam/beam.py:430-458 (numpy mean / std over the
 * particles with id != 0; id may be NULL: all alive).  Writes 8 doubles to
 * the device array stats: n_alive, mean_dt, sigma_dt, mean_dE, sigma_dE,
 * epsn_rms_l = pi sigma_dE sigma_dt, sum dt^2, sum dE^2.  stats also holds the
 * previous call's means, used as the shift of the one-pass sums (NaN or
 * zeros are fine on the first call).  scratch: BLOND_STATS_SCRATCH doubles,
 * ticket: one int that must be 0 before the first call (it is 0 again after
 * every call); calls sharing them must not overlap on the device. */
#define BLOND_STATS_MAX_BLOCKS 1024
#define BLOND_STATS_SCRATCH (7 * BLOND_STATS_MAX_BLOCKS)
int blond_beam_statistics_f64(const double* dt, const double* dE,
                              const int64_t* id, int64_t n, double* stats,
                              double* scratch, int* ticket, void* stream);
int blond_beam_statistics_f32(const float* dt, const float* dE,
                              const int64_t* id, int64_t n, double* stats,
                              double* scratch, int* ticket, void* stream);

/* ------------------------------------------------------------ cut limits
 * replaces the automatic frame of CutOptions.set_cuts() beam/profile.py:185-195
 * (cut_left and cut_right both None).  Writes 2 doubles to the device array
 * cuts: n_sigma <= 0 (the reference's None): dt_min - 0.05 (dt_max - dt_min)
 * and dt_max + 0.05 (dt_max - dt_min), bit-identical to the reference (min
 * and max are exact, the expressions are evaluated in its order); n_sigma > 0:
 * mean -/+ n_sigma sigma / 2 with numpy's mean and population std, to
 * rounding (~1e-16 relative).  NaN in dt gives NaN cuts, as numpy.  The _f32
 * variant reads float dt and evaluates in float64.  scratch:
 * BLOND_STATS_SCRATCH doubles, ticket: one int that is 0 before the first
 * call (0 again after every call). */
int blond_cut_limits_f64(const double* dt, int64_t n, double n_sigma, double* cuts,
                         double* scratch, int* ticket, void* stream);
int blond_cut_limits_f32(const float* dt, int64_t n, double n_sigma, double* cuts,
                         double* scratch, int* ticket, void* stream);

/* ------------------------------------------------------------ impedance setup
 * replaces fast_resonator_real_imag() cpp_routines/fast_resonator.cpp:19-74
 * re/im accumulate (+= / -=); index 0 (DC) is untouched. */
int blond_fast_resonator_f64(double* re, double* im, const double* freq,
                             const double* R_S, const double* Q,
                             const double* freq_R, int n_resonators,
                             int64_t n_freq, void* stream);

/* ------------------------------------------------------------ FFT
 * numpy.fft.rfft(x, n_fft) / numpy.fft.irfft(X, n_fft) as used by
 * bmath_backends.py:447-449 (Profile.beam_spectrum_generation,
 * profile.py:899-903; _InducedVoltage.induced_voltage_1turn,
 * impedance.py:475-485).  Complex arrays are interleaved (re, im) doubles.
 * n_fft must be even, 2..131072, with no prime factor above 5 (every
 * next_regular() result qualifies), or any length <= 4096 (direct DFT). */
int blond_rfft_f64(const double* x, int64_t n_x, int64_t n_fft,
                   double* spectrum, void* stream);
int blond_irfft_f64(const double* spectrum, int64_t n_fft, double* y,
                    int64_t n_out, void* stream);

/* One-turn induced voltage from the FFT path (impedance.py:457-489 with the
 * truncation of TotalInducedVoltage.induced_voltage_sum, impedance.py:113-131):
 *   v_out[k] = -scale * irfft(impedance * rfft(profile, n_fft), n_fft)[k]
 * for k < n_out, scale = charge * e * ratio; impedance holds n_fft/2+1
 * complex values (already divided by bin_size, impedance.py:889). */
int blond_induced_voltage_f64(const double* profile, int n_slices,
                              const double* impedance, int64_t n_fft,
                              double scale, double* v_out, int64_t n_out,
                              void* stream);

/* ------------------------------------------------------------ time-domain wakes
 * Analytic resonator convolution of InducedVoltageResonator: replaces
 * resonator_induced_voltage_1_turn() utils/butils_wrap_python.py:656-790
 * (called from InducedVoltageResonator.induced_voltage_1turn,
 * impedances/impedance.py:1286-1315).  For each time_array[j]:
 *   tmp_matrix[r][j] = R_S[r] / (2 omega_R[r] Q[r])
 *                      * sum_k kappa_k (F_r(t_j - bc_{k+1}) - F_r(t_j - bc_k)),
 *   induced_voltage[j] = scale * sum_r tmp_matrix[r][j],
 * kappa_k = (n_macroparticles[k+1] - n_macroparticles[k])
 *           / (bc_{k+1} - bc_k) / (beam_n_macroparticles * bin_size),
 * F_r as the reference defines it, scale = -charge * e * beam_n_macroparticles
 * * ratio.  The sum is evaluated by a recurrence over the bins in O(n_slices)
 * per resonator plus O(log n_slices) per time point, which needs the
 * n_slices bin_centers strictly increasing (a Profile's always are) and
 * agrees with the reference's O(n_time * n_slices) sum to rounding: about
 * 1e-13 of max|V| inside the slicing window, and within the reference's own
 * phase rounding (a * t_j in double) beyond it.
 *   - n_macroparticles, bin_centers, time_array, induced_voltage (n_time),
 *     tmp_matrix (n_resonators x n_time, row-major; may be NULL) and
 *     workspace are device arrays; R_S, omega_R and Q are HOST arrays.
 *   - workspace holds blond_resonator_workspace_bytes(n_slices,
 *     n_resonators) bytes, 16-byte aligned; the outputs must not overlap it.
 *   - 1 <= n_resonators <= BLOND_MAX_RESONATORS, 1 <= n_slices <= 2^24,
 *     Q >= 0.5 (the reference's constructor raises for Q < 0.5,
 *     impedance.py:1127-1129) and omega_R > 0, else an error code. */
#define BLOND_MAX_RESONATORS 64
int64_t blond_resonator_workspace_bytes(int n_slices, int n_resonators);
int blond_resonator_induced_voltage_f64(
    const double* n_macroparticles, const double* bin_centers, int n_slices,
    double bin_size, double beam_n_macroparticles, const double* time_array,
    int64_t n_time, const double* R_S, const double* omega_R, const double* Q,
    int n_resonators, double scale, double* induced_voltage, double* tmp_matrix,
    void* workspace, int64_t workspace_bytes, void* stream);

/* One turn of InducedVoltageResonator's multi-turn memory
 * (impedances/impedance.py:1317-1335) fused with the convolution above:
 *   memory_out[j] = memory_in[j + shift] (0 past n_memory)
 *                   + induced_voltage[j] (j < n_time),   j < n_memory,
 * where induced_voltage is what blond_resonator_induced_voltage_f64 gives
 * (the reference appends `shift` = n_slices zeros, drops the first
 * n_slices points and adds the new voltage to the first n_time).
 * memory_in and memory_out are distinct device arrays of n_memory >= n_time
 * doubles; the other arguments as above. */
int blond_resonator_mtw_f64(
    const double* n_macroparticles, const double* bin_centers, int n_slices,
    double bin_size, double beam_n_macroparticles, const double* time_array,
    int64_t n_time, const double* R_S, const double* omega_R, const double* Q,
    int n_resonators, double scale, const double* memory_in, double* memory_out,
    int64_t n_memory, int64_t shift, double* tmp_matrix, void* workspace,
    int64_t workspace_bytes, void* stream);

/* numpy.interp(x + x_shift, xp, fp, left, right) on the device: bm.interp
 * (utils/bmath_backends.py:373) as _InducedVoltage.shift_trev_time uses it
 * for the multi-turn-wake memory (impedances/impedance.py:533-550).  flags
 * bit 0: use `left` below xp[0] (else fp[0]); bit 1: use `right` above
 * xp[m-1] (else fp[m-1]).  xp increasing; x, xp, fp, out device arrays; out
 * must not overlap xp or fp.  Bit-identical to numpy's loop (no FMA). */
int blond_interp_f64(const double* x, int64_t n, double x_shift,
                     const double* xp, const double* fp, int m, double left,
                     double right, int flags, double* out, void* stream);

/* ------------------------------------------------------------ fused turn engine
 * One object per beam.  A turn is, in the order of the reference main loop
 * [TotalInducedVoltage, RingAndRFTracker, Profile]
 * (__EXAMPLES/main_files/EX_05_Wake_impedance.py:318-339):
 *   induced voltage from the current profile -> linear_interp_kick (acc 0)
 *   -> RF kick (turn t) -> drift (turn t+1 parameters) -> slice_beam.
 * It replaces RingAndRFTracker.track() (trackers/tracker.py:521-615),
 * Profile.track() (beam/profile.py:700-719) and TotalInducedVoltage.track()
 * (impedances/impedance.py:133-146) for one beam, as two kernels per turn
 * replayed from a CUDA graph.  The turn counter lives on the device. */
typedef struct blond_engine blond_engine;

int blond_engine_create(blond_engine** engine, int precision, int n_rf,
                        int solver, int n_slices);
int blond_engine_destroy(blond_engine* engine);
/* host arrays over turns; column t of the reference's F-ordered
 * [n_rf, n_turns+1] programmes is voltage[t*n_rf .. t*n_rf+n_rf-1]
 * (rf_parameters.py:317-328).  acc_kick has n_turns entries
 * (= -RFStation.delta_E). */
int blond_engine_set_rf(blond_engine* engine, int64_t n_turns,
                        const double* voltage, const double* omega_rf,
                        const double* phi_rf, const double* acc_kick,
                        double charge);
/* host arrays of n_turns+1 entries (Ring/RFStation per-turn values). */
int blond_engine_set_drift(blond_engine* engine, double length_ratio,
                           double alpha_order, const double* t_rev,
                           const double* eta_0, const double* eta_1,
                           const double* eta_2, const double* alpha_0,
                           const double* alpha_1, const double* alpha_2,
                           const double* beta, const double* energy);
/* bin_centers: host, n_slices values exactly as Profile.bin_centers. */
int blond_engine_set_slicing(blond_engine* engine, double cut_left,
                             double cut_right, const double* bin_centers);
/* FFT impedance (host, interleaved complex, n_fft/2+1 values, the sum of
 * every InducedVoltageFreq/Time total_impedance with this n_fft);
 * scale = charge * e * ratio. */
int blond_engine_set_impedance(blond_engine* engine, int64_t n_fft,
                               const double* impedance, double scale);
/* InductiveImpedance (impedance.py:986-1009): host z_over_n[n_turns+1];
 * scale = charge * e / (2 pi) * ratio; uses t_rev from set_drift. */
int blond_engine_set_inductive(blond_engine* engine, const double* z_over_n,
                               double scale);
/* dt/dE: device arrays of n macro-particles in the engine's precision
 * (F64: both double; F32P64: dt double, dE float; Q32P64: dt double, dE
 * int32 counts of the energy unit). */
int blond_engine_bind_beam(blond_engine* engine, void* dt, void* dE,
                           int64_t n);
/* No counterpart in the reference (its energies are floating point).
 * Q32P64 only, required before tracking: eV per count of the int32 dE.
 * Every turn's energy change is formed in float64 and rounded once to a
 * multiple of this unit; the grid spans +-(2^31 - 1) units, and a particle
 * leaving it is reported by blond_engine_check as BLOND_ERR_RANGE. */
int blond_engine_set_energy_unit(blond_engine* engine, double lsb);
/* RingAndRFTracker(interpolation=True) (trackers/tracker.py:586-601): each
 * turn's head interpolates the RF voltage at the bin centres (rf_volt_comp,
 * kick.cpp:37-51) plus the induced voltage, with the turn's acceleration
 * kick in the offsets (linear_interp_kick.cpp:44-47), and the particle pass
 * applies that one interpolated kick instead of the RF kick.  on = 0/1.
 * Not with the SPS_RL beam-phase loop, nor with another loop unless there
 * is an FFT impedance. */
int blond_engine_set_interpolation(blond_engine* engine, int on);
/* Profile with OtherSlicesOptions(smooth=True) (beam/profile.py:764-773):
 * each turn ends with a deposit pass of the reference's slice_smooth
 * weights (histogram.cpp:75-132) accumulated in 64-bit fixed point (2^-b
 * per unit weight, b = min(52, 62 - ceil(log2(1.5 n + 2))); the same bits
 * every run), which is the profile the next turn's induced voltage uses.
 * on = 0/1.  Not with a beam-phase loop or a bound (sharded) histogram. */
int blond_engine_set_smooth(blond_engine* engine, int on);
int blond_engine_set_turn(blond_engine* engine, int64_t turn, void* stream);
/* Re-slice the bound beam into the profile (Profile.track()). */
int blond_engine_slice(blond_engine* engine, void* stream);
/* Capture and upload the CUDA graph of turns_per_graph turns now (it is
 * otherwise built by the first blond_engine_run that needs it). */
int blond_engine_prepare(blond_engine* engine, void* stream);
/* Track n_turns fused turns; afterwards the profile holds the slices of the
 * final coordinates. */
int blond_engine_run(blond_engine* engine, int64_t n_turns, void* stream);
/* Synchronise `stream` and report a device-side failure of the runs so far:
 * BLOND_ERR_TIMEOUT if a bounded wait in a kernel gave up (the coordinates
 * are then not valid), BLOND_ERR_RANGE if a Q32P64 energy left its grid
 * (saturated there), else BLOND_OK.  Clears the flag. */
int blond_engine_check(blond_engine* engine, void* stream);

/* The beam-phase loop inside the turn: replaces BeamFeedback.track()
 * (llrf/beam_feedback.py:237-622) called by RingAndRFTracker.track()
 * (trackers/tracker.py:551-552) and the tracker's accumulation of the RF
 * phase offset (tracker.py:553-565), with no host work per turn.  In turn t
 * (turn >= delay) the beam phase of the profile is measured (beam_phase,
 * exp(alpha t)-weighted from time_offset on; SPS_F: the sharp window), the
 * machine's loop runs on device state and the frequency correction is added
 * to omega_rf of turn t + 1 of every RF system (times h_j / h_0); then, every
 * turn, dphi_rf += 2 pi h (omega_rf - omega_rf_d) / omega_rf_d at t + 1 and
 * phi_rf[t + 1] += dphi_rf.  With an FFT impedance the measurement is part
 * of the head kernel (its last CTA runs the loop), else one all-SM pass
 * converts the histogram and runs it.  SPS_RL also averages dE[::sample_dE]
 * of the bound beam (after the induced-voltage kick when there is an
 * impedance, as the reference's main loop orders it): one extra pass.
 *   turn_table: HOST, (n_turns + 1) rows of 11 + 2 n_rf values: phi_s, eta_0,
 *     alpha_0, gamma, beta, energy, lhc_a, lhc_t, PL gain, second gain,
 *     third gain (PSB radial integral), omega_rf_d[n_rf], harmonic[n_rf].
 *   state: HOST, BLOND_FB_STATE(n_rf) values: lhc_y, dphi_sum, dphi_av,
 *     dphi_av_prev, domega_PL, domega_RL, dR_over_R_prev, PL_counter,
 *     phi_beam, dphi, domega_rf, drho, dR_over_R, average_dE, (2 unused),
 *     dphi_rf[n_rf].
 *   on_time: HOST, the PSB loop's action turns (precalculate_time).
 * machine 0 removes the loop.  Phase noise is not modelled. */
#define BLOND_FB_LHC 1
#define BLOND_FB_LHC_F 2
#define BLOND_FB_SPS_F 3
#define BLOND_FB_SPS_RL 4
#define BLOND_FB_PSB 5
#define BLOND_FB_STATE(n_rf) (16 + (n_rf))
int blond_engine_set_feedback(blond_engine* engine, int machine, int delay,
                              double gain, double gain2, double alpha,
                              int has_time_offset, double time_offset,
                              double bin_size, double ring_radius,
                              int sample_dE, const double* turn_table,
                              const double* on_time, int n_on_time,
                              const double* state);
/* Device copies of the loop state, the omega_rf / phi_rf programmes
 * (turn-major, (n_turns + 1) x n_rf) and the per-turn trace ((n_turns + 1)
 * x 3: phi_beam, dphi, domega_rf); NULL skips an output. */
int blond_engine_get_feedback(blond_engine* engine, double* state,
                              double* omega_rf, double* phi_rf, double* trace,
                              void* stream);
/* Particle-pass implementation: 0 = bulk-copy (TMA) pipelined (default;
 * falls back to 1 when the profile is too long for its shared memory),
 * 1 = plain loads, 3 = plain loads with a packed 16-bit block histogram
 * (up to 2^17 slices beside the prefetch ring; needs an interpolated kick),
 * 2 = plain loads with the interpolation table in shared
 * memory (the induced voltage for F64 / Q32P64, entries formed per particle
 * with the head's rounding) and a packed 16-bit histogram; 2 needs an FFT
 * impedance, a non-interpolated kick, integer slicing, bin centres that are
 * numpy.linspace midpoints of the cuts, and the shared memory for it
 * (BLOND_ERR_UNSUPPORTED otherwise). */
int blond_engine_set_kernel(blond_engine* engine, int variant);
/* Device copies of the current state (n_slices doubles each). */
int blond_engine_get_profile(blond_engine* engine, double* profile,
                             void* stream);
int blond_engine_get_induced_voltage(blond_engine* engine, double* v,
                                     void* stream);
int blond_engine_get_turn(blond_engine* engine, int64_t* turn_host);
/* Track n_turns like blond_engine_run but without a graph, bracketing each
 * of the two launches of every turn with CUDA events on `stream`; returns
 * the summed device durations of the head and particle kernels (ms) and
 * synchronises the stream.  Measurement only. */
int blond_engine_time_kernels(blond_engine* engine, int64_t n_turns,
                              double* head_ms, double* particles_ms,
                              void* stream);
/* Sharded tracking (one beam split over several GPUs; the exchange is the
 * reference's MPI Profile.reduce_histo, beam/profile.py:721-762): bind a caller-
 * owned int32 histogram of n_slices counts (NULL restores the engine's
 * own), then drive the turns step by step and sum the histogram over the
 * ranks (e.g. an NCCL all-reduce) after every particle step:
 *   slice; all-reduce; step(3)              -- initial profile
 *   repeat: step(1); step(2); all-reduce    -- one turn
 *   step(3)                                 -- profile of the final turn
 * part 1 = head (profile, induced voltage, table; clears the histogram),
 * part 2 = particle pass of the current turn (advances the turn),
 * part 3 = profile <- histogram. */
/* Turns on coordinates in HOST memory (host_dt doubles, host_dE of the
 * engine's precision, n particles each; page-locked memory lets the copies
 * overlap).  Each turn copies the beam to the bound device arrays, runs the
 * turn and copies it back, in `chunks` pieces pipelined against the
 * particle pass (in and out copies on two streams).  The caller's stream
 * completes after the last copy. */
int blond_engine_track_host(blond_engine* engine, double* host_dt, void* host_dE,
                            int64_t n_turns, int chunks, void* stream);
int blond_engine_bind_histogram(blond_engine* engine, int* hist);
int blond_engine_step(blond_engine* engine, int part, void* stream);
/* Grid size and block size of the particle kernel (0 = automatic). */
int blond_engine_tune(blond_engine* engine, int threads, int blocks_per_sm,
                      int turns_per_graph);
/* Histogram layout of the particle pass: -1 automatic, 0 block-private
 * ints with warp-aggregated deposits, 1 block-private ints, 2 block-private
 * packed 16-bit counters (staged pass), 3 global-memory atomics (plain
 * pass).  A layout that does not fit falls back to the automatic one. */
int blond_engine_set_histogram(blond_engine* engine, int mode);
/* Plain pass: depth of the per-thread cp.async prefetch ring (0 = direct
 * loads, 2 or 4 stages). */
int blond_engine_set_prefetch(blond_engine* engine, int stages);
/* Shared-table pass: thread 0 of each block also prefetches the block's
 * slice one iteration beyond the ring into L2 (cp.async.bulk.prefetch);
 * on = 0/1. */
int blond_engine_set_l2_prefetch(blond_engine* engine, int on);
/* Programmatic dependent launch between a turn's kernels (default on):
 * each kernel lets the next one launch and run its prologue before the
 * previous one's results are visible; on = 0 launches them in plain stream
 * order.  The results are the same either way. */
int blond_engine_set_overlap(blond_engine* engine, int on);
/* Plain pass: blocks (1, 2, 4, 8) of a thread-block cluster whose shared
 * histograms are summed through distributed shared memory before one
 * global flush per cluster. */
int blond_engine_set_cluster(blond_engine* engine, int blocks);
/* Autotuner: times every feasible particle-pass configuration (plain pass:
 * 256/512/1024 threads x 1/2/4 blocks per SM x histogram layouts x prefetch
 * ring 0/2/4 x clusters of 1/2; staged pass: histogram layouts; shared-table
 * pass: ring 0/2; packed-histogram pass: ring 0/2/4) on the bound beam,
 * `reps` (1..10) launches each after one warm-up, and keeps the fastest;
 * then replays a few whole turns with and without programmatic dependent
 * launch (blond_engine_set_overlap) and keeps the faster (not with a
 * beam-phase loop or smooth slicing).  Restores the coordinates, the
 * histogram, the turn counter, the induced voltage and the profile.
 * config[9] receives {variant (0 staged, 1 plain, 2 shared table,
 * 3 packed histogram), threads, blocks per SM, histogram
 * layout, ring stages, cluster blocks, L2 prefetch (0/1), candidates
 * timed, overlap (0/1)}; best_ms the
 * particle-pass time of the winner.  Not inside stream capture; allocates
 * a snapshot of the coordinates for the duration of the call. */
int blond_engine_autotune(blond_engine* engine, int reps, void* stream, int* config,
                          double* best_ms);

/* ------------------------------------------------------------ batched beams
 * Many independent beams (one RingAndRFTracker + Profile +
 * TotalInducedVoltage each in the reference) tracked together: one
 * particle launch and one head launch per turn for the whole batch, each
 * beam with its own particle count, RF programme, slicing window and
 * impedance, and the single-beam engine's arithmetic.  Host arrays are
 * beam-major: RF [B][n_turns+1][n_rf], acc [B][n_turns], drift arrays
 * [B][n_turns+1], cuts [B], bin_centers [B][n_slices], impedance
 * [B][n_fft/2+1] complex, scale [B] (= charge * e * ratio of each beam).
 * dt/dE: device arrays of all beams concatenated, beam b occupying
 * [offsets[b], offsets[b+1]) (host offsets), both 16-byte aligned (the
 * particle pass loads neighbouring particles in pairs). */
typedef struct blond_batch blond_batch;
int blond_batch_create(blond_batch** batch, int precision, int n_beams, int n_rf,
                       int solver, int n_slices);
int blond_batch_destroy(blond_batch* batch);
int blond_batch_set_rf(blond_batch* batch, int64_t n_turns, const double* voltage,
                       const double* omega_rf, const double* phi_rf,
                       const double* acc_kick, double charge);
int blond_batch_set_drift(blond_batch* batch, double length_ratio, double alpha_order,
                          const double* t_rev, const double* eta_0, const double* eta_1,
                          const double* eta_2, const double* alpha_0, const double* alpha_1,
                          const double* alpha_2, const double* beta, const double* energy);
int blond_batch_set_slicing(blond_batch* batch, const double* cut_left,
                            const double* cut_right, const double* bin_centers);
int blond_batch_set_impedance(blond_batch* batch, int64_t n_fft, const double* impedance,
                              const double* scale);
int blond_batch_bind_beams(blond_batch* batch, void* dt, void* dE, const int64_t* offsets);
/* No counterpart in the reference.  Q32P64 only, required before tracking:
 * host array of B energy units (eV per count of each beam's int32 dE), as
 * blond_engine_set_energy_unit. */
int blond_batch_set_energy_units(blond_batch* batch, const double* lsb);
/* Synchronise `stream`; BLOND_ERR_RANGE if a Q32P64 energy left its beam's
 * grid since the last check, else BLOND_OK.  Clears the flag. */
int blond_batch_check(blond_batch* batch, void* stream);
/* Launch shape of the particle pass: threads per block (multiple of 32,
 * <= 1024), blocks per SM, particles per thread and iteration (2, 4, 8),
 * chunk (particles of one block's piece of a beam, 1024..2^22) and
 * warp-aggregated shared-memory deposits (0/1).  Default 512, 2, 4, 32768,
 * 0.  The reference's GPU backend uses one fixed grid for every kernel
 * (blond/gpu/__init__.py:47-50). */
int blond_batch_set_shape(blond_batch* batch, int threads, int blocks_per_sm,
                          int particles_per_thread, int chunk, int aggregate);
/* Time every launch shape above on the bound beams (CUDA events; the
 * coordinates and histograms are restored) and keep the fastest.
 * config (host, 6 ints) = {threads, blocks_per_sm, particles_per_thread,
 * chunk, aggregate, candidates tried}; best_ms = its particle pass. */
int blond_batch_autotune(blond_batch* batch, int reps, void* stream, int* config,
                         double* best_ms);
int blond_batch_set_turn(blond_batch* batch, int64_t turn, void* stream);
int blond_batch_slice(blond_batch* batch, void* stream);
/* capture and upload the turn graph now (else the first long run does) */
int blond_batch_prepare(blond_batch* batch, void* stream);
int blond_batch_run(blond_batch* batch, int64_t n_turns, void* stream);
int blond_batch_tune(blond_batch* batch, int turns_per_graph);
/* device outputs of B * n_slices doubles (beam-major) */
int blond_batch_get_profiles(blond_batch* batch, double* profiles, void* stream);
int blond_batch_get_induced_voltages(blond_batch* batch, double* v, void* stream);

/* ------------------------------------------------------------ one turn, no allocation
 * No counterpart in the reference.  One fused turn of the engine -- slice
 * the input coordinates, induced voltage (when `impedance` is not NULL) and
 * its interpolated kick, RF kick, drift, slice -- for callers that must not
 * allocate device memory: a tracking step embedded in a host application
 * that owns the device's memory (an online model, a framework with its own
 * pooling allocator) cannot call cudaMalloc, which may stall the whole
 * device and bypasses the host's accounting.  Nothing is allocated: the
 * temporaries live in a fixed file-scope device array of ~448 KB that every
 * device loading the library holds until the process exits.  The array is
 * committed when the library's device code is loaded on a device; with
 * CUDA's lazy module loading (the default) that happens in the first call.
 *   - n_slices <= 16384, else BLOND_ERR_SIZE; n_fft as for the engine.
 *   - dt, dE, voltage, omega_rf, phi_rf, impedance (n_fft/2+1 complex,
 *     16-byte aligned), profile_out and induced_voltage_out (n_slices
 *     doubles) are device arrays.  Drift scalars are this turn's drift
 *     parameters (turn+1 values in the reference tracker), voltage/
 *     omega_rf/phi_rf this turn's RF column; beta and energy must be > 0.
 *   - The bin centres are those of the reference's Profile for the cuts:
 *     the midpoints of numpy.linspace(cut_left, cut_right, n_slices + 1),
 *     computed on the device with numpy's operations.
 *   - The first call on a device looks the scratch up
 *     (cudaGetSymbolAddress) and sets kernel attributes: make it before
 *     any stream capture.  Every call only enqueues kernels on `stream`
 *     (no copies, no synchronisation).
 *   - Every call shares the scratch: calls that overlap on the GPU (two
 *     streams, two threads) race.  Each call clears the histogram it
 *     starts from. */
int blond_turn_f64_noalloc(double* dt, double* dE, int64_t n, int n_rf,
                           double charge, const double* voltage,
                           const double* omega_rf, const double* phi_rf,
                           double acc_kick, int solver, double t_rev,
                           double length_ratio, double alpha_order,
                           double eta_0, double eta_1, double eta_2,
                           double alpha_0, double alpha_1, double alpha_2,
                           double beta, double energy, double cut_left,
                           double cut_right, int n_slices,
                           const double* impedance, int64_t n_fft,
                           double iv_scale, double* profile_out,
                           double* induced_voltage_out, void* stream);

/* ------------------------------------------------------------ adjoint segment
 * No counterpart in the reference (it has no derivatives).  The building
 * blocks of a differentiable N-turn map -- profile by cloud-in-cell
 * deposition, induced voltage, interpolated kick, RF kick, simple drift --
 * and of its adjoint, driven turn by turn by a host that checkpoints the
 * coordinates every K turns (blond_b200/adjoint.py).  Coordinates are
 * device arrays: dt double, dE double (BLOND_PREC_F64) or float
 * (BLOND_PREC_F32P64); adjoints are double.  The bin grid is the profile's
 * bin centres bin_center0 + k / inv_bin_width, k < n_slices; cloud-in-cell
 * gives a particle at f = (dt - bin_center0) * inv_bin_width the weight
 * 1 - (f - floor f) in bin floor f and the rest in the next bin.
 * voltage / omega_rf / phi_rf point at this turn's n_rf (<= 4) device
 * values; drift_coeff = t_rev length_ratio eta_0 / (beta^2 E) of turn + 1. */

/* profile (n_slices zeros on entry) = cloud-in-cell deposit of dt, with
 * weights rounded to multiples of 2^-b, b = min(52, 62 - ceil(log2(n+1))),
 * so that every run gives the same bits (integer accumulation, independent
 * of the order of the atomics) */
int blond_adjoint_deposit(const double* dt, int64_t n, int n_slices, double bin_center0,
                          double inv_bin_width, double* profile, void* stream);
/* one forward turn: induced_voltage (n_slices values, or NULL) kick,
 * RF kick, drift, then profile_out (zeros on entry, or NULL: none) = the
 * deposit of the new dt as above; dt_out / dE_out may alias dt_in / dE_in */
int blond_adjoint_forward_turn(int precision, const double* dt_in, const void* dE_in,
                               double* dt_out, void* dE_out, int64_t n, int n_rf,
                               const double* voltage, const double* omega_rf,
                               const double* phi_rf, double acc_kick, double charge,
                               double drift_coeff, const double* induced_voltage,
                               int n_slices, double bin_center0, double inv_bin_width,
                               double* profile_out, void* stream);
/* one backward turn.  On entry lam_dt / lam_dE hold dL/d(dt, dE) at turn
 * t+1 and lam_p_next dL/d(profile at turn t+1) (deposited at dt_next, or
 * NULL); on exit they hold dL/d(dt, dE) at turn t excluding the turn-t
 * profile.  lam_v += dL/d(induced voltage of turn t); grad_rf[j] +=
 * dL/dV_j and grad_rf[n_rf + j] += dL/dphi_j of this turn.  kick = 0 only
 * adds the deposit adjoint of lam_p_next at dt_next. */
int blond_adjoint_backward_turn(const double* dt, const double* dt_next, int64_t n,
                                double* lam_dt, double* lam_dE, const double* lam_p_next,
                                int kick, int n_rf, const double* voltage,
                                const double* omega_rf, const double* phi_rf, double charge,
                                double drift_coeff, const double* induced_voltage,
                                int n_slices, double bin_center0, double inv_bin_width,
                                double* lam_v, double* grad_rf, void* stream);
/* mode 0: y = -scale irfft(Z rfft(x, n_fft))[:n_slices] (the induced
 *         voltage), spectrum (n_fft/2+1 complex, or NULL) = rfft(x, n_fft);
 * mode 1: the transpose, with impedance = conj(Z):
 *         y = -scale irfft(conj(Z) rfft(x))[:n_slices], and
 *         accum[k] += spectrum[k] conj(rfft(x)[k]).
 * Cluster transform lengths only (even 5-smooth n_fft <= 131072). */
int blond_adjoint_spectral(int mode, const double* x, int n_slices, const double* impedance,
                           int64_t n_fft, double scale, double* y, double* spectrum,
                           double* accum, void* stream);
/* The forward map's turn loop in one call: profile[0] = deposit of dt, then
 * for t < n_turns: every checkpoint_every turns a copy of (dt, dE) into row
 * t / checkpoint_every of ckpt_dt / ckpt_dE; with an impedance (n_fft/2+1
 * complex, or NULL) induced_voltage[t] and spectrum[t] from profile[t]
 * (mode 0 above); one forward turn into profile[t + 1].  voltage, omega_rf,
 * phi_rf: device [n_turns][n_rf]; acc_kick, drift_coeff: HOST [n_turns];
 * profile: device [n_turns + 1][n_slices], zeros on entry. */
int blond_adjoint_forward_run(int precision, double* dt, void* dE, int64_t n, int n_rf,
                              int64_t n_turns, const double* voltage, const double* omega_rf,
                              const double* phi_rf, const double* acc_kick,
                              const double* drift_coeff, double charge,
                              const double* impedance, int64_t n_fft, double scale,
                              double* induced_voltage, double* spectrum, double* profile,
                              int n_slices, double bin_center0, double inv_bin_width,
                              int checkpoint_every, double* ckpt_dt, void* ckpt_dE,
                              void* stream);
/* The backward sweep in one call: segment by segment from the last, the
 * segment's turn-start dt recomputed from its checkpoint into states
 * ([checkpoint_every + 1][n]; dE_work [n] holds the energies), then the
 * backward turns (with an impedance, conj(Z) as impedance_conj: lam_v[t]
 * through mode 1 above into lam_pt[t], accumulating spectrum_accum), and
 * last the deposit adjoint of the turn-0 profile.  lam_p_final: dL/d(final
 * profile) or NULL.  On exit lam_dt / lam_dE hold dL/d(initial dt, dE),
 * grad_rf[t] = {dL/dV_j, dL/dphi_j}. */
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
                               double* spectrum_accum, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BLOND_B200_H */
