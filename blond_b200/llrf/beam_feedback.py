"""BeamFeedback: one-turn beam-phase loop (blond/llrf/beam_feedback.py:35-648).

The loop's input, the beam phase, is a reduction over the profile and runs
on the device (blond_beam_phase_f64 / _f32, one block); the loop filters
are scalar recurrences per turn and run on the host as in the reference,
which then corrects omega_rf[:, turn + 1].  RingAndRFTracker calls track()
at the start of every turn >= delay and re-sends the changed omega_rf
column.

Machines: 'LHC' (phase + synchro loop), 'LHC_F' (phase + frequency loop),
'SPS_F' (sharp-window beam phase + frequency loop), 'SPS_RL' (phase +
radial loop), 'PSB' (phase and radial loops acting once per sampling
period).  Phase noise objects are used through their ``dphi`` array and an
LHCNoiseFB-like object through its ``x`` attribute, as the reference does.
"""
from __future__ import annotations

import numpy as np

from .. import bmath as bm


class BeamFeedback:
    def __init__(self, ring, rf_station, profile, configuration, PhaseNoise=None,
                 LHCNoiseFB=None, delay: int = 0):
        self.ring = ring
        self.rf_station = rf_station
        self.profile = profile
        self.config = configuration
        self.delay = delay
        self.machine = self.config.get("machine", "LHC")
        self.alpha = self.config.get("window_coefficient", 0.0)
        self.time_offset = self.config.get("time_offset", None)
        if "PL_gain" not in self.config:
            raise RuntimeError("You need to specify the Phase Loop gain! Aborting")
        self.gain = self.config["PL_gain"]
        n1 = rf_station.n_turns + 1
        if self.machine == "LHC":
            self.gain2 = self.config.get("SL_gain", 0.0)
            self.lhc_y = 0
            if self.gain2 != 0:
                # synchro-loop coefficient a and time constant tau per turn
                # (beam_feedback.py:95-110)
                self.lhc_a = 5.25 - self.rf_station.omega_s0 / (np.pi * 40.0)
                self.lhc_t = ((2 * np.pi * self.rf_station.Q_s * np.sqrt(self.lhc_a))
                              / np.sqrt(1 + self.gain / self.gain2
                                        * np.sqrt((1 + 1 / self.lhc_a)
                                                  / (1 + self.lhc_a))))
            else:
                self.lhc_a = np.zeros(n1)
                self.lhc_t = np.zeros(n1)
        elif self.machine in ("LHC_F", "SPS_F"):
            self.gain2 = self.config.get("FL_gain", 0.0)
        elif self.machine == "SPS_RL":
            self.gain2 = self.config.get("RL_gain", 0.0)
            self.sample_dE = self.config.get("sample_dE", 1)
        elif self.machine == "PSB":
            self.gain = self.gain * np.ones(ring.n_turns + 1)
            # the reference scales the configuration's own list in place
            self.gain2 = self.config.get("RL_gain", [0.0, 0.0])
            self.gain2[0] = self.gain2[0] * np.ones(ring.n_turns + 1)
            self.gain2[1] = self.gain2[1] * np.ones(ring.n_turns + 1)
            self.dt = self.config.get("period", 10.0e-6)
            self.PL_counter = 0
            self.on_time = np.array([])
            self.precalculate_time(ring)
            self.coefficients = self.config.get(
                "coefficients", [0.999019, -0.999019, 0.0, 1.0, -0.998038, 0.0])
            self.dphi_sum = 0.0
            self.dphi_av = 0.0
            self.dphi_av_prev = 0.0
            self.dR_over_R_prev = 0.0
            self.domega_PL = 0.0
            self.domega_RL = 0.0
            self.dR_over_R = 0
        self.drho = 0.0
        self.domega_rf = 0.0
        self.phi_beam = 0.0
        self.dphi = 0.0
        self.reference = 0.0
        self.RFnoise = PhaseNoise
        if self.RFnoise is not None and len(self.RFnoise.dphi) != ring.n_turns + 1:
            raise RuntimeError("Phase noise has to have a length of n_turns + 1")
        self.noiseFB = LHCNoiseFB

    # ----------------------------------------------------------------- turn
    def track(self):
        """beam_feedback.py:237-254: this machine's correction, applied to
        next turn's frequency of every RF system in proportion to its
        harmonic."""
        getattr(self, self.machine)()
        rf = self.rf_station
        nxt = rf.counter[0] + 1
        rf.omega_rf[:, nxt] += self.domega_rf * rf.harmonic[:, nxt] / rf.harmonic[0, nxt]

    def precalculate_time(self, ring):
        """beam_feedback.py:256-274: the turns on which the PSB loops act,
        the last turn of every `period` seconds of revolution time after
        `delay`; a trailing 0 where the programme ends inside a period."""
        if self.dt <= 0:
            self.on_time = np.arange(ring.t_rev.size)
            return
        turns = []
        n = self.delay + 1
        while n < ring.t_rev.size:
            elapsed = 0
            while elapsed < self.dt:
                if n >= ring.t_rev.size:
                    self.on_time = np.append(np.array(turns, dtype=float), 0)
                    return
                elapsed += ring.t_rev[n]
                n += 1
            turns.append(n - 1)
        self.on_time = np.array(turns, dtype=float)

    # ----------------------------------------------------------- measures
    def _rf_now(self):
        t = self.rf_station.counter[0]
        return float(self.rf_station.omega_rf[0, t]), float(self.rf_station.phi_rf[0, t])

    def _bin_range(self, lo=None, hi=None):
        """Indices [start, stop) of the increasing bin centres within
        [lo, hi]: a contiguous run, the bins the reference's boolean masks
        select."""
        bc = np.asarray(self.profile.bin_centers)
        start = 0 if lo is None else int(np.searchsorted(bc, lo, side="left"))
        stop = bc.size if hi is None else int(np.searchsorted(bc, hi, side="right"))
        return start, max(start, stop)

    def beam_phase(self):
        """beam_feedback.py:276-309: exp(alpha t)-windowed projections of the
        line density (bins from time_offset on) at the main RF frequency,
        reduced on the device; the phase is arctan of their ratio + pi."""
        omega_rf, phi_rf = self._rf_now()
        start, stop = self._bin_range(self.time_offset, None)
        coeff = bm.beam_phase(self.profile.bin_centers_dev, self.profile.n_macroparticles,
                              self.alpha, omega_rf, phi_rf, self.profile.bin_size,
                              start=start, stop=stop)
        self.phi_beam = np.arctan(coeff) + np.pi

    def beam_phase_sharpWindow(self):
        """beam_feedback.py:311-347: unweighted projections over the bins of
        a window set by alpha and time_offset (all bins when alpha is 0)."""
        omega_rf, phi_rf = self._rf_now()
        if self.alpha != 0.0:
            lo = self.time_offset - np.pi / omega_rf
            hi = -1 / self.alpha + self.time_offset - 2 * np.pi / omega_rf
            start, stop = self._bin_range(lo, hi)
        else:
            start, stop = 0, int(self.profile.n_slices)
        coeff = bm.beam_phase_fast(self.profile.bin_centers_dev,
                                   self.profile.n_macroparticles, omega_rf, phi_rf,
                                   self.profile.bin_size, start=start, stop=stop)
        self.phi_beam = np.arctan(coeff) + np.pi

    def phase_difference(self):
        """beam_feedback.py:349-368."""
        counter = self.rf_station.counter[0]
        self.dphi = self.phi_beam - self.rf_station.phi_s[counter]
        if self.RFnoise is not None:
            if self.noiseFB is not None:
                self.dphi += self.noiseFB.x * self.RFnoise.dphi[counter]
            elif self.machine != "PSB":
                self.dphi += self.RFnoise.dphi[counter]

    def radial_difference(self):
        """beam_feedback.py:370-391: relative radial offset from the mean
        energy of every sample_dE-th particle (a device reduction)."""
        counter = self.rf_station.counter[0]
        dE = self.profile.beam.dE[:: self.sample_dE]
        self.average_dE = float(dE.double().mean())
        self.drho = (self.ring.alpha_0[0, counter] * self.ring.ring_radius
                     * self.average_dE
                     / (self.ring.beta[0, counter] ** 2.0 * self.ring.energy[0, counter]))

    def radial_steering_from_freq(self):
        """beam_feedback.py:393-430.  The reference accumulates into
        rf_station.dphi_rf_steering, which nothing defines, so a non-zero
        `reference` fails there with AttributeError; it does here too."""
        rf = self.rf_station
        counter = rf.counter[0]
        self.radial_steering_domega_rf = (-rf.omega_rf_d[0, counter] * rf.eta_0[counter]
                                          / self.ring.alpha_0[0, counter] * self.reference
                                          / self.ring.ring_radius)
        rf.omega_rf[:, counter] += (self.radial_steering_domega_rf * rf.harmonic[:, counter]
                                    / rf.harmonic[0, counter])
        rf.dphi_rf_steering += (2.0 * np.pi * rf.harmonic[:, counter]
                                * (rf.omega_rf[:, counter] - rf.omega_rf_d[:, counter])
                                / rf.omega_rf_d[:, counter])
        rf.phi_rf[:, counter] += rf.dphi_rf_steering

    # ------------------------------------------------------------ machines
    def LHC_F(self):
        """beam_feedback.py:432-458: phase loop + frequency loop."""
        counter = self.rf_station.counter[0]
        self.beam_phase()
        self.phase_difference()
        self.domega_rf = -self.gain * self.dphi - self.gain2 * (
            self.rf_station.omega_rf[0, counter] - self.rf_station.omega_rf_d[0, counter]
            + self.reference)

    def SPS_F(self):
        """beam_feedback.py:460-479: LHC_F with the sharp-window phase."""
        counter = self.rf_station.counter[0]
        self.beam_phase_sharpWindow()
        self.phase_difference()
        self.domega_dphi = -self.gain * self.dphi
        self.domega_df = -self.gain2 * (self.rf_station.omega_rf[0, counter]
                                        - self.rf_station.omega_rf_d[0, counter])
        self.domega_rf = self.domega_dphi + self.domega_df

    def SPS_RL(self):
        """beam_feedback.py:481-514: phase loop + radial loop."""
        counter = self.rf_station.counter[0]
        if self.reference != 0:
            self.radial_steering_from_freq()
        self.beam_phase()
        self.phase_difference()
        self.radial_difference()
        self.domega_dphi = -self.gain * self.dphi
        self.domega_dR = (-np.sign(self.rf_station.eta_0[counter]) * self.gain2
                          * (self.reference - self.drho) / self.ring.ring_radius)
        self.domega_rf = self.domega_dphi + self.domega_dR

    def LHC(self):
        """beam_feedback.py:516-565: phase loop + synchro loop with its
        recursion y <- (1 - tau) y + (1 - a) tau (dphi_rf + reference)."""
        counter = self.rf_station.counter[0]
        dphi_rf = self.rf_station.dphi_rf[0]
        self.beam_phase()
        self.phase_difference()
        self.domega_rf = -self.gain * self.dphi - self.gain2 * (
            self.lhc_y + self.lhc_a[counter] * (dphi_rf + self.reference))
        self.lhc_y = ((1 - self.lhc_t[counter]) * self.lhc_y
                      + (1 - self.lhc_a[counter]) * self.lhc_t[counter]
                      * (dphi_rf + self.reference))

    def PSB(self):
        """beam_feedback.py:567-622: the phase error averaged between
        sampling turns drives the phase loop's filter; the radial loop acts
        on the relative frequency offset."""
        counter = self.rf_station.counter[0]
        self.beam_phase()
        self.phase_difference()
        self.dphi_sum += self.dphi
        if counter == self.on_time[self.PL_counter] and counter >= self.delay:
            self.dphi_av = self.dphi_sum / (self.on_time[self.PL_counter]
                                            - self.on_time[self.PL_counter - 1])
            if self.RFnoise is not None:
                self.dphi_av += self.RFnoise.dphi[counter]
            self.domega_PL = 0.99803799 * self.domega_PL + self.gain[counter] * (
                0.99901903 * self.dphi_av - 0.99901003 * self.dphi_av_prev)
            self.dphi_av_prev = self.dphi_av
            self.dphi_sum = 0.0
            rf = self.rf_station
            self.dR_over_R = (rf.omega_rf[0, counter] - rf.omega_rf_d[0, counter]) / (
                rf.omega_rf_d[0, counter]
                * (1.0 / (self.ring.alpha_0[0, counter] * rf.gamma[counter] ** 2) - 1.0))
            self.domega_RL = (self.domega_RL
                              + self.gain2[0][counter] * (self.dR_over_R - self.dR_over_R_prev)
                              + self.gain2[1][counter] * self.dR_over_R)
            self.dR_over_R_prev = self.dR_over_R
            self.PL_counter += 1
        self.domega_rf = -self.domega_PL - self.domega_RL

    def to_gpu(self, recursive=True):
        self._device = "GPU"

    def to_cpu(self, recursive=True):
        self._device = "CPU"
