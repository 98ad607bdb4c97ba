"""RingAndRFTracker: RF kick and drift per turn (blond/trackers/tracker.py:263-615).

``track()`` follows the reference step by step: phase-noise update, the
dphi_rf accumulation of the RF phase (host, O(n_rf)), then either the
multi-harmonic kick or -- with ``interpolation=True`` -- the RF voltage over
the bin centres plus the induced voltage applied by linear interpolation,
then the drift with the turn+1 parameters, on the device coordinates.  The
RF programme is uploaded to the device once (turn-major, one contiguous
column per turn); only a phase column that dphi_rf changed is re-sent.
The beam-phase loop (``beam_feedback``, blond_b200.llrf.BeamFeedback) runs
at the start of every turn >= its delay and corrects next turn's omega_rf
column, which is re-sent.  Noise and cavity feedback, periodicity and
xsuite coupling are not supported.
"""
from __future__ import annotations

import numpy as np
import torch

from .. import bmath as bm


class RingAndRFTracker:
    def __init__(self, rf_station, beam, solver: str = "simple",
                 beam_feedback=None, noise_feedback=None, cavity_feedback=None,
                 periodicity: bool = False, interpolation: bool = False,
                 with_xsuite: bool = False, profile=None,
                 total_induced_voltage=None):
        if noise_feedback is not None or cavity_feedback is not None:
            raise NotImplementedError("noise and cavity feedback are not supported")
        if periodicity or with_xsuite:
            raise NotImplementedError("periodicity / xsuite are not supported")
        self.rf_params = rf_station
        self.counter = rf_station.counter
        self.acceleration_kick = -rf_station.delta_E
        self.beam = beam
        self.solver = str(solver)
        if self.solver not in ("simple", "exact", "legacy"):
            raise RuntimeError("ERROR in RingAndRFTracker: Choice of longitudinal "
                               "solver not recognised!")
        if self.rf_params.alpha_order > 1:
            self.solver = "exact"
        self.beamFB = beam_feedback
        self.noiseFB = self.cavityFB = None
        self.periodicity = False
        self.with_xsuite = False
        self.interpolation = bool(interpolation)
        self.profile = profile
        self.totalInducedVoltage = total_induced_voltage
        if self.interpolation and self.profile is None:
            raise RuntimeError("ERROR in RingAndRFTracker: Please specify a "
                               "Profile object to use the interpolation option")
        self._dev_prog = None

    # ------------------------------------------------------------ programme
    def _programme(self):
        """Device copies (turn-major) of voltage, omega_rf and phi_rf."""
        dtype = self.beam.dt.dtype
        if self._dev_prog is None or self._dev_prog[0].dtype != dtype:
            rf = self.rf_params
            self._dev_prog = tuple(
                torch.as_tensor(np.ascontiguousarray(np.asarray(a, float).T),
                                device=self.beam.dt.device).to(dtype)
                for a in (rf.voltage, rf.omega_rf, rf.phi_rf))
        return self._dev_prog

    def kick(self, beam_dt, beam_dE, index: int):
        """tracker.py:399-422."""
        V, om, ph = self._programme()
        bm.kick(beam_dt, beam_dE, V[index], om[index], ph[index],
                self.rf_params.particle.charge, self.rf_params.n_rf,
                self.acceleration_kick[index])

    def drift(self, beam_dt, beam_dE, index: int):
        """tracker.py:424-468."""
        rf = self.rf_params
        bm.drift(beam_dt, beam_dE, self.solver, rf.t_rev[index], rf.length_ratio,
                 rf.alpha_order, rf.eta_0[index], rf.eta_1[index], rf.eta_2[index],
                 rf.alpha_0[index], rf.alpha_1[index], rf.alpha_2[index],
                 rf.beta[index], rf.energy[index])

    def rf_voltage_calculation(self):
        """tracker.py:470-519 (no cavity feedback)."""
        t = self.counter[0]
        V, om, ph = self._programme()
        self.rf_voltage = bm.rf_volt_comp(V[t], om[t], ph[t],
                                          self.profile.bin_centers_dev)

    def track(self):
        """tracker.py:521-615."""
        turn = self.counter[0]
        rf = self.rf_params
        if rf.phi_noise is not None:
            rf.phi_rf[:, turn] += rf.phi_noise[:, turn]
            self._sync_phase(turn)
        if self.beamFB is not None and turn >= self.beamFB.delay:
            self.beamFB.track()
            self._sync_column(1, turn + 1)
        rf.dphi_rf += (2.0 * np.pi * rf.harmonic[:, turn + 1]
                       * (rf.omega_rf[:, turn + 1] - rf.omega_rf_d[:, turn + 1])
                       / rf.omega_rf_d[:, turn + 1])
        if np.any(rf.dphi_rf != 0):
            rf.phi_rf[:, turn + 1] += rf.dphi_rf
            self._sync_phase(turn + 1)
        if not rf.empty:
            if self.interpolation:
                self.rf_voltage_calculation()
                if self.totalInducedVoltage is not None:
                    self.total_voltage = self.rf_voltage + \
                        self.totalInducedVoltage.induced_voltage
                else:
                    self.total_voltage = self.rf_voltage
                bm.linear_interp_kick(self.beam.dt, self.beam.dE, self.total_voltage,
                                      self.profile.bin_centers_dev,
                                      self.beam.particle.charge,
                                      self.acceleration_kick[turn])
            else:
                self.kick(self.beam.dt, self.beam.dE, turn)
        self.drift(self.beam.dt, self.beam.dE, turn + 1)
        self.beam.beta = float(rf.beta[turn + 1])
        self.beam.gamma = float(rf.gamma[turn + 1])
        self.beam.energy = float(rf.energy[turn + 1])
        self.beam.momentum = float(rf.momentum[turn + 1])
        self.counter[0] += 1

    def _sync_phase(self, t: int):
        self._sync_column(2, t)

    def _sync_column(self, which: int, t: int):
        """Re-send turn t of omega_rf (which=1) or phi_rf (which=2)."""
        if self._dev_prog is not None:
            src = (self.rf_params.omega_rf, self.rf_params.phi_rf)[which - 1]
            col = torch.as_tensor(np.asarray(src[:, t], float))
            self._dev_prog[which][t].copy_(col.to(self._dev_prog[which].dtype))


class FullRingAndRF:
    """RingAndRFTracker sections tracked in order (trackers/tracker.py:
    60-213); the potential-well helpers are not provided."""

    def __init__(self, ring_and_rf_section):
        self.ring_and_rf_section = list(ring_and_rf_section)
        self.ring_circumference = 0.0
        for section in self.ring_and_rf_section:
            self.ring_circumference += section.rf_params.section_length
        self.ring_radius = self.ring_circumference / (2 * np.pi)

    def track(self):
        for section in self.ring_and_rf_section:
            section.track()
