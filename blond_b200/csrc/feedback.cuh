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
    const void* dE;
    int dE_f32;
    int64_t n;
    double* partials;  // kFbPartials doubles
    double* om;        // RF programmes, turn-major [t * n_rf + j]
    double* ph;
    const double* table;  // (n_turns + 1) x (FB_COLS + 2 n_rf)
    const double* on_time;
    int n_on_time;
    double* state;
    double* trace;  // (n_turns + 1) x 3: phi_beam, dphi, domega_rf
    int64_t n_turns;
};

constexpr int kFbPartials = 296;  // blocks of the dE reduction (2 per SM on B200)

int launch_feedback(const FeedbackArgs& a, cudaStream_t s);

}  // namespace bb
