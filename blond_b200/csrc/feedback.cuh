// The beam-phase loop run inside the fused engine's turn (feedback.cu):
// after the head kernel of turn t has written the profile, one block
// measures the beam phase, runs the machine's loop filter on device-resident
// state and corrects the RF programme of turn t + 1, as
// BeamFeedback.track() and RingAndRFTracker.track() do on the host
// (llrf/beam_feedback.py:237-622, trackers/tracker.py:551-565).
#pragma once

#include "common.cuh"

namespace bb {

// columns of the per-turn table (turn-major, FB_COLS + 2 n_rf per turn)
enum {
    FBT_PHI_S, FBT_ETA0, FBT_ALPHA0, FBT_GAMMA, FBT_BETA, FBT_ENERGY, FBT_LHC_A, FBT_LHC_T,
    FBT_GAIN, FBT_GAIN2A, FBT_GAIN2B, FB_COLS  // then omega_rf_d[n_rf], harmonic[n_rf]
};
// device state (doubles); dphi_rf[n_rf] follows FBS_DPHI_RF
enum {
    FBS_LHC_Y, FBS_DPHI_SUM, FBS_DPHI_AV, FBS_DPHI_AV_PREV, FBS_DOMEGA_PL, FBS_DOMEGA_RL,
    FBS_DR_PREV, FBS_PL_COUNTER, FBS_PHI_BEAM, FBS_DPHI, FBS_DOMEGA_RF, FBS_DRHO, FBS_DR,
    FBS_AVG_DE, FBS_DPHI_RF = 16
};

struct FeedbackArgs {
    int machine;  // BLOND_FB_*
    int delay, n_rf;
    long long* turn;  // the head has already advanced it: this turn is *turn - 1
    const double* profile;
    const double* bc;
    int S;
    double bin_size;
    double alpha, time_offset;
    int has_time_offset;
    double gain, gain2, ring_radius;
    // SPS_RL: mean of dE[::sample_dE] over the bound beam
    int sample_dE;
    const double* dt;
    const void* dE;
    int dE_f32;
    int64_t n;
    double* partials;        // kFbPartials doubles (the dE sums)
    double* phase_partials;  // 2 kFbMaxParts doubles (the beam-phase warp sums)
    double* om;        // RF programmes, turn-major [t * n_rf + j]
    double* ph;
    const double* table;  // (n_turns + 1) x (FB_COLS + 2 n_rf)
    const double* on_time;
    int n_on_time;
    double* state;
    double* trace;  // (n_turns + 1) x 3: phi_beam, dphi, domega_rf
    int64_t n_turns;
};

constexpr int kFbPartials = 1184;  // blocks of the dE reductions (8 per SM on B200)
constexpr int kFbThreads = 256;    // threads per block of the convert kernel
constexpr int kFbMaxBlocks = 148;  // at most one block per SM
constexpr int kFbMaxParts = 1024;  // warp partials of the beam phase (phase_partials / 2)
constexpr int kFbMaxRf = 16;       // RF systems (the engine's limit)

// SPS_RL: the dE partial sums the loop averages (before the loop's turn).
int launch_feedback_dE(const FeedbackArgs& a, cudaStream_t s);
// SPS_RL after an induced-voltage head: the dE partial sums with this
// turn's interpolated kick applied (the reference averages dE after
// TotalInducedVoltage.track); table as the particle pass reads it.
int launch_feedback_dE_lik(const FeedbackArgs& a, const void* table, double bc0,
                           double lik_inv_w, double bw, cudaStream_t s);
// The loop of this turn in one pass: histogram -> profile (histogram
// cleared) with the beam-phase sums, the last block running the loop; bump
// advances the turn counter afterwards (heads without a spectral kernel).
// With hist == nullptr the profile the head wrote is read instead (the turn
// counter already advanced).
int launch_feedback_turn(const FeedbackArgs& a, int* hist, int* ticket, int bump,
                         cudaStream_t s);

#ifdef __CUDACC__
// The bins the beam phase integrates: [lo, hi] on the bin centres.  SPS_F
// (beam_phase_sharpWindow, beam_feedback.py:326-334) cuts a window from
// alpha and time_offset when alpha != 0; the other machines (beam_phase,
// :287-306) take every bin from time_offset on.
struct FbBins {
    const double* bc;
    int S, machine;
    double alpha, lo, hi, omega, phi;
};

__device__ __forceinline__ FbBins fb_bins(const FeedbackArgs& a, long long t) {
    FbBins b;
    b.bc = a.bc;
    b.S = a.S;
    b.machine = a.machine;
    b.alpha = a.alpha;
    b.omega = a.om[(size_t)t * a.n_rf];
    b.phi = a.ph[(size_t)t * a.n_rf];
    b.lo = -INFINITY;
    b.hi = INFINITY;
    if (b.machine == BLOND_FB_SPS_F) {
        if (b.alpha != 0.0) {
            b.lo = a.time_offset - M_PI / b.omega;
            b.hi = -1 / b.alpha + a.time_offset - 2 * M_PI / b.omega;
        }
    } else if (a.has_time_offset) {
        b.lo = a.time_offset;
    }
    return b;
}

// Bin i's terms of the two projections (beam_phase.cpp:6-40) with its
// trapezoid weight within the window (trapz_const_delta,
// blondmath.cpp:496-512): 1 inside, 1/2 at either end, 1 for a window of
// one bin, 0 outside.
__device__ __forceinline__ void fb_add(const FbBins& b, int i, double x, double& s_sum,
                                       double& c_sum) {
    const double bci = b.bc[i];
    if (!(b.lo <= bci && bci <= b.hi)) return;
    const bool first = i == 0 || !(b.lo <= b.bc[i - 1]);
    const bool last = i == b.S - 1 || !(b.bc[i + 1] <= b.hi);
    const double w = (first && last) ? 1.0 : ((first || last) ? 0.5 : 1.0);
    const double base = b.machine != BLOND_FB_SPS_F ? exp(b.alpha * bci) * x : x;
    double sn, cs;
    sincos(b.omega * bci + b.phi, &sn, &cs);
    s_sum += w * (base * sn);
    c_sum += w * (base * cs);
}

// The loop of turn t from the summed projections (one thread): phase,
// machine filter, next turn's frequency correction, phase accumulation,
// trace.  Its scalar inputs are read together up front through the
// read-only path, so the chain is one round of loads, not one per value.
__device__ __forceinline__ void fb_turn_end(const FeedbackArgs& a, long long t, double s_sum,
                                            double c_sum, double d_sum) {
    const int nr = a.n_rf;
    const int cols = FB_COLS + 2 * nr;
    const double* __restrict__ row = a.table + (size_t)t * cols;
    const double* __restrict__ nxt = a.table + (size_t)(t + 1) * cols;
    double* __restrict__ st = a.state;
    double* __restrict__ om1 = a.om + (size_t)(t + 1) * nr;
    double* __restrict__ ph1 = a.ph + (size_t)(t + 1) * nr;
    const double omega = __ldg(a.om + (size_t)t * nr);
    const double phi_s = __ldg(row + FBT_PHI_S), eta0 = __ldg(row + FBT_ETA0);
    const double alpha0 = __ldg(row + FBT_ALPHA0), gamma = __ldg(row + FBT_GAMMA);
    const double beta = __ldg(row + FBT_BETA), energy = __ldg(row + FBT_ENERGY);
    const double la = __ldg(row + FBT_LHC_A), lt = __ldg(row + FBT_LHC_T);
    const double gain_t = __ldg(row + FBT_GAIN), g2a = __ldg(row + FBT_GAIN2A);
    const double g2b = __ldg(row + FBT_GAIN2B), od0 = __ldg(row + FB_COLS);
    const double h0n = __ldg(nxt + FB_COLS + nr);
    double lhc_y = __ldg(st + FBS_LHC_Y), dphi_sum = __ldg(st + FBS_DPHI_SUM);
    double dphi_av = __ldg(st + FBS_DPHI_AV), dphi_av_prev = __ldg(st + FBS_DPHI_AV_PREV);
    double domega_pl = __ldg(st + FBS_DOMEGA_PL), domega_rl = __ldg(st + FBS_DOMEGA_RL);
    double dr_prev = __ldg(st + FBS_DR_PREV), pl_counter = __ldg(st + FBS_PL_COUNTER);
    double phi_beam = __ldg(st + FBS_PHI_BEAM), dphi = __ldg(st + FBS_DPHI);
    double domega = __ldg(st + FBS_DOMEGA_RF), drho = __ldg(st + FBS_DRHO);
    double dr = __ldg(st + FBS_DR), avg = __ldg(st + FBS_AVG_DE);
    const double dphi_rf0 = __ldg(st + FBS_DPHI_RF);
    const bool active = t >= a.delay;
    if (active) {
        // coefficient of beam_phase.cpp; the phase projected to (pi/2, 3pi/2)
        const double coeff = (a.bin_size * s_sum) / (a.bin_size * c_sum);
        phi_beam = atan(coeff) + M_PI;
        dphi = phi_beam - phi_s;           // phase_difference, :349-368
        const double om_off = omega - od0;  // omega_rf - omega_rf_d, main system
        switch (a.machine) {
        case BLOND_FB_LHC:  // beam_feedback.py:516-565
            domega = -a.gain * dphi - a.gain2 * (lhc_y + la * (dphi_rf0 + 0.0));
            lhc_y = (1 - lt) * lhc_y + (1 - la) * lt * (dphi_rf0 + 0.0);
            break;
        case BLOND_FB_LHC_F:  // beam_feedback.py:432-458
            domega = -a.gain * dphi - a.gain2 * (om_off + 0.0);
            break;
        case BLOND_FB_SPS_F:  // beam_feedback.py:460-479
            domega = -a.gain * dphi + -a.gain2 * om_off;
            break;
        case BLOND_FB_SPS_RL: {  // beam_feedback.py:370-391, 481-514
            const int64_t m = (a.n + a.sample_dE - 1) / a.sample_dE;
            avg = d_sum / (double)m;
            drho = alpha0 * a.ring_radius * avg / (beta * beta * energy);
            const double sgn = eta0 > 0 ? 1.0 : (eta0 < 0 ? -1.0 : 0.0);
            domega = -a.gain * dphi + -sgn * a.gain2 * (0.0 - drho) / a.ring_radius;
            break;
        }
        case BLOND_FB_PSB: {  // beam_feedback.py:567-622
            dphi_sum += dphi;
            const int pc = (int)pl_counter;
            if (pc < a.n_on_time && (double)t == a.on_time[pc]) {
                const double prev = a.on_time[pc > 0 ? pc - 1 : a.n_on_time - 1];
                dphi_av = dphi_sum / (a.on_time[pc] - prev);
                domega_pl = 0.99803799 * domega_pl +
                            gain_t * (0.99901903 * dphi_av - 0.99901003 * dphi_av_prev);
                dphi_av_prev = dphi_av;
                dphi_sum = 0.0;
                dr = om_off / (od0 * (1.0 / (alpha0 * (gamma * gamma)) - 1.0));
                domega_rl = domega_rl + g2a * (dr - dr_prev) + g2b * dr;
                dr_prev = dr;
                pl_counter = pc + 1;
            }
            domega = -domega_pl - domega_rl;
            break;
        }
        }
    }
    // BeamFeedback.track (:237-254): next turn's frequency of every system,
    // then RingAndRFTracker.track (tracker.py:553-565): accumulated phase
    // offset, added to next turn's phase when any is non-zero
    bool any = false;
    for (int j = 0; j < nr; ++j) {
        double o = om1[j];
        const double od = __ldg(nxt + FB_COLS + j), h = __ldg(nxt + FB_COLS + nr + j);
        if (active) o += domega * h / h0n;
        om1[j] = o;
        const double d = st[FBS_DPHI_RF + j] + 2.0 * M_PI * h * (o - od) / od;
        st[FBS_DPHI_RF + j] = d;
        any = any || d != 0.0;
    }
    if (any)
        for (int j = 0; j < nr; ++j) ph1[j] += st[FBS_DPHI_RF + j];
    st[FBS_LHC_Y] = lhc_y;
    st[FBS_DPHI_SUM] = dphi_sum;
    st[FBS_DPHI_AV] = dphi_av;
    st[FBS_DPHI_AV_PREV] = dphi_av_prev;
    st[FBS_DOMEGA_PL] = domega_pl;
    st[FBS_DOMEGA_RL] = domega_rl;
    st[FBS_DR_PREV] = dr_prev;
    st[FBS_PL_COUNTER] = pl_counter;
    st[FBS_PHI_BEAM] = phi_beam;
    st[FBS_DPHI] = dphi;
    st[FBS_DOMEGA_RF] = domega;
    st[FBS_DRHO] = drho;
    st[FBS_DR] = dr;
    st[FBS_AVG_DE] = avg;
    if (a.trace) {
        a.trace[t * 3 + 0] = phi_beam;
        a.trace[t * 3 + 1] = dphi;
        a.trace[t * 3 + 2] = domega;
    }
}

#endif  // __CUDACC__

}  // namespace bb
