"""Induced voltage from impedances (blond/impedances/impedance.py:47-1009).

Per turn the hot step is ``-(q e ratio) irfft(Z rfft(profile, n_fft))``,
which here is ONE cluster launch (blond_induced_voltage_f64) for every
even 5-smooth n_fft, followed by the interpolated kick.  Impedance set-up
(resonator impedance, wake spectra) also runs on the device.  Multi-turn
wakes are not supported (multi_turn_wake=True raises).
"""
from __future__ import annotations

import numpy as np
import torch
from scipy.constants import e

from .. import bmath as bm
from ..toolbox.next_regular import next_regular


def induced_voltage_lengths(n_slices: int, bin_size: float, cut_left: float,
                            cut_right: float, wake_length=None,
                            frequency_resolution=None):
    """(n_induced_voltage, wake_length) as _InducedVoltage.process
    (impedance.py:349-403) derives them."""
    if wake_length is not None and frequency_resolution is None:
        n_iv = int(np.ceil(wake_length / bin_size))
        if n_iv < n_slices:
            raise RuntimeError("Error: too short wake length. Increase it above "
                               f"{n_slices * bin_size:1.2e} s.")
        return n_iv, n_iv * bin_size
    if frequency_resolution is not None and wake_length is None:
        n_iv = int(np.ceil(1 / (bin_size * frequency_resolution)))
        if n_iv < n_slices:
            raise RuntimeError("Error: too large frequency_resolution. Reduce it "
                               f"below {1 / (cut_right - cut_left):1.2e} Hz.")
        return n_iv, n_iv * bin_size
    if wake_length is None and frequency_resolution is None:
        return n_slices, cut_right - cut_left
    raise RuntimeError("Error: only one of wake_length or frequency_resolution "
                       "can be specified.")


def _smooth_even(n: int) -> bool:
    if n < 2 or n % 2:
        return False
    m = n // 2
    for f in (2, 3, 5):
        while m % f == 0:
            m //= f
    return m == 1 and n <= 131072


class TotalInducedVoltage:
    """Sum of the induced voltages and the kick they give
    (impedance.py:47-146)."""

    def __init__(self, beam, profile, induced_voltage_list):
        self.beam = beam
        self.profile = profile
        self.induced_voltage_list = induced_voltage_list
        self.induced_voltage = torch.zeros(int(profile.n_slices),
                                           dtype=profile.n_macroparticles.dtype,
                                           device="cuda")
        self.time_array = profile.bin_centers

    def reprocess(self):
        for obj in self.induced_voltage_list:
            obj.process()

    def induced_voltage_sum(self):
        spectra = {}
        total = 0
        for obj in self.induced_voltage_list:
            obj.induced_voltage_generation(spectra)
            total = total + obj.induced_voltage[: self.profile.n_slices]
        self.induced_voltage = total.to(self.profile.n_macroparticles.dtype).contiguous()

    def track(self):
        self.induced_voltage_sum()
        bm.linear_interp_kick(self.beam.dt, self.beam.dE, self.induced_voltage,
                              self.profile.bin_centers_dev,
                              self.beam.particle.charge, 0.0)


class _InducedVoltage:
    def __init__(self, beam, profile, frequency_resolution=None, wake_length=None,
                 multi_turn_wake: bool = False, mtw_mode="time", rf_station=None,
                 use_regular_fft: bool = True):
        if multi_turn_wake:
            raise NotImplementedError("multi-turn wakes are not supported")
        self.beam = beam
        self.profile = profile
        self.wake_length_input = wake_length
        self.frequency_resolution_input = frequency_resolution
        self.use_regular_fft = use_regular_fft
        self.rf_params = rf_station
        self.multi_turn_wake = False
        self.mtw_mode = mtw_mode
        self.n_fft = None
        self.total_impedance = None
        self.induced_voltage = torch.zeros(int(profile.n_slices),
                                           dtype=profile.n_macroparticles.dtype,
                                           device="cuda")
        self.process()

    def process(self):
        self.n_induced_voltage, self.wake_length = induced_voltage_lengths(
            self.profile.n_slices, self.profile.bin_size, self.profile.cut_left,
            self.profile.cut_right, self.wake_length_input,
            self.frequency_resolution_input)
        self.induced_voltage_generation = self.induced_voltage_1turn

    def _scale(self) -> float:
        return self.beam.particle.charge * e * self.beam.ratio

    def induced_voltage_1turn(self, beam_spectrum_dict=None):
        """impedance.py:457-489."""
        dtype = self.profile.n_macroparticles.dtype
        if _smooth_even(self.n_fft):
            v = bm.induced_voltage_1turn(self.profile.n_macroparticles,
                                         self.total_impedance, self.n_fft,
                                         self._scale(), self.n_induced_voltage)
        else:
            if beam_spectrum_dict is None:
                beam_spectrum_dict = {}
            if self.n_fft not in beam_spectrum_dict:
                self.profile.beam_spectrum_generation(self.n_fft)
                beam_spectrum_dict[self.n_fft] = self.profile.beam_spectrum
            y = bm.irfft(self.total_impedance * beam_spectrum_dict[self.n_fft])
            v = -(self._scale() * y)[: self.n_induced_voltage]
        self.induced_voltage = v.to(dtype)


class InducedVoltageTime(_InducedVoltage):
    """Induced voltage from wakes (impedance.py:575-697)."""

    def __init__(self, beam, profile, wake_source_list, wake_length=None,
                 multi_turn_wake: bool = False, rf_station=None, mtw_mode="time",
                 use_regular_fft: bool = True):
        self.wake_source_list = wake_source_list
        self.total_wake = 0
        _InducedVoltage.__init__(self, beam, profile, frequency_resolution=None,
                                 wake_length=wake_length,
                                 multi_turn_wake=multi_turn_wake,
                                 rf_station=rf_station, mtw_mode=mtw_mode,
                                 use_regular_fft=use_regular_fft)

    def process(self):
        _InducedVoltage.process(self)
        n = int(self.n_induced_voltage) + int(self.profile.n_slices) - 1
        self.n_fft = next_regular(n) if self.use_regular_fft else n
        self.frequency_resolution = 1 / (self.n_fft * self.profile.bin_size)
        self.time = np.arange(0, self.wake_length,
                              self.wake_length / self.n_induced_voltage,
                              dtype=bm.precision.real_t)
        self.sum_wakes(self.time)

    def sum_wakes(self, time_array):
        self.total_wake = np.zeros(time_array.shape)
        for w in self.wake_source_list:
            w.wake_calc(time_array)
            self.total_wake += w.wake
        self.total_impedance = bm.rfft(self.total_wake, self.n_fft)


class InducedVoltageFreq(_InducedVoltage):
    """Induced voltage from impedances (impedance.py:700-890)."""

    def __init__(self, beam, profile, impedance_source_list,
                 frequency_resolution=None, multi_turn_wake: bool = False,
                 front_wake_length: float = 0, rf_station=None, mtw_mode="time",
                 use_regular_fft: bool = True):
        self.impedance_source_list = impedance_source_list
        self.total_impedance = 0
        self.front_wake_length = front_wake_length
        self.freq = None
        self.frequency_resolution = None
        _InducedVoltage.__init__(self, beam, profile, wake_length=None,
                                 frequency_resolution=frequency_resolution,
                                 multi_turn_wake=multi_turn_wake,
                                 rf_station=rf_station, mtw_mode=mtw_mode,
                                 use_regular_fft=use_regular_fft)

    def process(self):
        _InducedVoltage.process(self)
        self.n_fft = next_regular(self.n_induced_voltage) if self.use_regular_fft \
            else self.n_induced_voltage
        self.profile.beam_spectrum_freq_generation(self.n_fft)
        self.freq = self.profile.beam_spectrum_freq
        self.frequency_resolution = 1 / (self.n_fft * self.profile.bin_size)
        if self.front_wake_length:
            self.front_wake_buffer = int(np.ceil(np.max(self.front_wake_length)
                                                 / self.profile.bin_size))
        self.sum_impedances(self.freq)

    def sum_impedances(self, freq):
        total = torch.zeros(len(freq), dtype=torch.complex128, device="cuda")
        for src in self.impedance_source_list:
            src.imped_calc(freq)
            total += src.impedance
        self.total_impedance = total / self.profile.bin_size


class InductiveImpedance(_InducedVoltage):
    """Constant imaginary Z/n (impedance.py:932-1009)."""

    def __init__(self, beam, profile, Z_over_n, rf_station,
                 deriv_mode: str = "gradient"):
        z = np.asarray(Z_over_n, dtype=float)
        if z.ndim == 0:
            z = np.full(rf_station.n_turns + 1, float(z))
        self.Z_over_n = z
        self.deriv_mode = deriv_mode
        _InducedVoltage.__init__(self, beam, profile, rf_station=rf_station)

    def induced_voltage_1turn(self, beam_spectrum_dict=None):
        index = self.rf_params.counter[0]
        coeff = -(self.beam.particle.charge * e / (2 * np.pi) * self.beam.ratio
                  * self.Z_over_n[index] * self.rf_params.t_rev[index]
                  / self.profile.bin_size)
        deriv = self.profile.beam_profile_derivative(self.deriv_mode)[1]
        v = coeff * deriv
        self.induced_voltage = v[: self.n_induced_voltage].to(
            self.profile.n_macroparticles.dtype)
