"""Induced voltage from impedances (blond/impedances/impedance.py:47-1009).

Per turn the hot step is ``-(q e ratio) irfft(Z rfft(profile, n_fft))``,
which here is ONE cluster launch (blond_induced_voltage_f64) for every
even 5-smooth n_fft, followed by the interpolated kick.  Impedance set-up
(resonator impedance, wake spectra) also runs on the device.

Multi-turn wakes (impedance.py:404-550) keep their memory on the device:
mtw_mode 'time' shifts it by one revolution period with the device
numpy.interp (blond_interp_f64), mtw_mode 'freq' by a phase ramp in the
frequency domain.  InducedVoltageResonator (impedance.py:1042-1377)
evaluates the analytic resonator convolution with
blond_resonator_induced_voltage_f64.
"""
from __future__ import annotations

import warnings

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
    """Base of the induced-voltage objects (impedance.py:190-572)."""

    def __init__(self, beam, profile, frequency_resolution=None, wake_length=None,
                 multi_turn_wake: bool = False, mtw_mode="time", rf_station=None,
                 use_regular_fft: bool = True):
        self.beam = beam
        self.profile = profile
        self.wake_length_input = wake_length
        self.frequency_resolution_input = frequency_resolution
        self.use_regular_fft = use_regular_fft
        self.rf_params = rf_station
        self.multi_turn_wake = bool(multi_turn_wake)
        if mtw_mode not in ("freq", "time"):
            raise ValueError(f"mtw_mode must be 'freq' or 'time', not {mtw_mode!r}")
        self.mtw_mode = mtw_mode
        self.n_fft = None
        self.total_impedance = None
        self.n_mtw_memory = None
        self.front_wake_buffer = None
        self.mtw_memory = None
        self.omegaj_mtw = None
        self.time_mtw = None
        self.induced_voltage = torch.zeros(int(profile.n_slices),
                                           dtype=profile.n_macroparticles.dtype,
                                           device="cuda")
        self.process()

    def process(self):
        """impedance.py:349-455."""
        self.n_induced_voltage, self.wake_length = induced_voltage_lengths(
            self.profile.n_slices, self.profile.bin_size, self.profile.cut_left,
            self.profile.cut_right, self.wake_length_input,
            self.frequency_resolution_input)
        if not self.multi_turn_wake:
            self.induced_voltage_generation = self.induced_voltage_1turn
            return
        self.n_mtw_memory = self.n_induced_voltage
        self.front_wake_buffer = 0
        bin_size = self.profile.bin_size
        if self.mtw_mode == "freq":
            # One revolution of buffer against the circular shift, plus the
            # object's buffer_extra (which the reference never sets either:
            # without it this raises AttributeError there too).
            self.buffer_size = np.ceil(np.max(self.rf_params.t_rev) / bin_size)
            self.buffer_size += np.ceil(np.max(self.buffer_extra) / bin_size)
            self.n_mtw_memory += int(self.buffer_size)
            self.n_mtw_fft = next_regular(self.n_mtw_memory) if self.use_regular_fft \
                else self.n_mtw_memory
            self.freq_mtw = bm.rfftfreq(self.n_mtw_fft, d=bin_size)
            self.omegaj_mtw = torch.as_tensor(2.0j * np.pi * self.freq_mtw,
                                              dtype=torch.complex128, device="cuda")
            self.shift_trev = self.shift_trev_freq
        else:
            self.shift_trev = self.shift_trev_time
            time_mtw = np.linspace(0, self.wake_length, self.n_mtw_memory,
                                   endpoint=False, dtype=bm.precision.real_t)
            self.time_mtw = torch.as_tensor(time_mtw.astype(np.float64), device="cuda")
        self.mtw_memory = torch.zeros(self.n_mtw_memory,
                                      dtype=self.profile.n_macroparticles.dtype,
                                      device="cuda")
        self.induced_voltage_generation = self.induced_voltage_mtw

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

    def induced_voltage_mtw(self, beam_spectrum_dict=None):
        """impedance.py:491-516: shift the memory by one turn, add this
        turn's voltage (its front-wake tail zeroed) and read it back."""
        self.shift_trev()
        self.induced_voltage_1turn(beam_spectrum_dict)
        n_iv = int(self.n_induced_voltage)
        v = self.induced_voltage
        if self.front_wake_buffer:
            v[n_iv - int(self.front_wake_buffer):] = 0
        self.mtw_memory[:n_iv] += v[:n_iv].to(self.mtw_memory.dtype)
        self.induced_voltage = self.mtw_memory[:n_iv]

    def _t_rev_now(self) -> float:
        return float(self.rf_params.t_rev[self.rf_params.counter[0]])

    def shift_trev_freq(self):
        """impedance.py:518-531: multiply the spectrum of the memory by
        exp(2 pi j f t_rev), back-transform, zero the last buffer_size
        points."""
        spec = bm.rfft(self.mtw_memory, self.n_mtw_fft)
        spec = spec * torch.exp(self.omegaj_mtw * self._t_rev_now())
        mem = bm.irfft(spec)[: self.n_mtw_memory].to(self.mtw_memory.dtype)
        mem[-int(self.buffer_size):] = 0
        self.mtw_memory = mem.contiguous()

    def shift_trev_time(self):
        """impedance.py:533-550: memory(t + t_rev) by linear interpolation
        on time_mtw, 0 outside it."""
        self.mtw_memory = bm.interp(self.time_mtw, self.time_mtw, self.mtw_memory,
                                    left=0, right=0, x_shift=self._t_rev_now()
                                    ).to(self.mtw_memory.dtype)


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


# resonators per launch of the convolution kernel (BLOND_MAX_RESONATORS)
_RESONATORS_PER_LAUNCH = 64


def mtw_resonator_time_array(bin_centers, n_slices: int, t_rev, n_turns: int,
                             min_index: int = 0) -> np.ndarray:
    """Times at which InducedVoltageResonator evaluates a multi-turn wake
    (impedance.py:1172-1193): for each turn k < n_turns the window
    linspace(bc_0, bc_last + 2 (bc_min_index - bc_0), n_slices + 2 min_index)
    moved by k t_rev[k]."""
    bc = np.asarray(bin_centers, dtype=np.float64)
    stop = bc[-1] + 2 * (bc[min_index] - bc[0])
    window = np.linspace(bc[0], stop, n_slices + 2 * min_index)
    parts = [t_rev[k] * k + window for k in range(n_turns)]
    return np.concatenate(parts) if parts else np.array([])


class InducedVoltageResonator(_InducedVoltage):
    """Induced voltage of resonators from the analytic convolution of the
    linearly interpolated line density (impedance.py:1042-1377), evaluated
    on the device by blond_resonator_induced_voltage_f64 in O(n_slices +
    n_time) per resonator.  With multi_turn_wake=True the times cover the
    turns over which the slowest mode decays to time_decay_factor (with the
    reference's own decay-turn formula, impedance.py:1159-1169) and the
    memory is shifted by one window per turn (impedance.py:1317-1335).

    Differences from the reference: the n_time x n_slices matrix _deltaT is
    never built (the attribute stays None), and for D < 0 beyond
    exp(-b D) = inf, where the reference returns NaN, this returns the
    Heaviside limit."""

    def __init__(self, beam, profile, resonators, frequency_resolution=None,
                 wake_length=None, multi_turn_wake: bool = False, mtw_mode="time",
                 rf_station=None, use_regular_fft: bool = True,
                 time_decay_factor=0.01, time_array=None):
        Q = np.asarray(resonators.Q, dtype=np.float64)
        if np.sum(Q < 0.5) > 0:
            raise RuntimeError("All quality factors Q must be larger than 0.5")
        if mtw_mode != "time":
            warnings.warn("InducedVoltageResonator only allows for 'time' mtw_mode, "
                          "'freq' will be ignored")
        if wake_length is not None:
            warnings.warn("InducedVoltageResonator ignores the setting of wake_length")
        if frequency_resolution is not None:
            warnings.warn("InducedVoltageResonator ignores the setting of "
                          "frequency_resolution")
        if not use_regular_fft:
            warnings.warn("use_regular_fft is not supported and will be ignored by "
                          "InducedVoltageResonator", UserWarning)
        self.beam = beam
        self.profile = profile
        omega_R = np.asarray(resonators.omega_R, dtype=np.float64)
        bc = np.asarray(profile.bin_centers, dtype=np.float64)
        if multi_turn_wake:
            if time_array is not None:
                warnings.warn("InducedVoltageResonator ignores time_array when "
                              "multi_turn_wake=True")
            decay_time = 2 * np.max(Q / omega_R)
            # the reference divides by log(e) with e the elementary charge
            decay_turns = np.ceil(np.log(time_decay_factor) / np.log(e) * decay_time
                                  / np.min(rf_station.t_rev))
            n_turns_calc = min(int(decay_turns), rf_station.n_turns)
            # argmin over a scalar difference: always 0, as in the reference
            potential_min_cav = rf_station.phi_s[0] / rf_station.omega_rf[0, 0]
            min_index = int(np.abs(bc[0] - potential_min_cav).argmin())
            self.time_array = mtw_resonator_time_array(
                bc, int(profile.n_slices), rf_station.t_rev, n_turns_calc, min_index)
            self.atLineDensityTimes = False
        elif time_array is None:
            self.time_array = profile.bin_centers
            self.atLineDensityTimes = True
        else:
            self.time_array = time_array
            self.atLineDensityTimes = False
        self.array_length = len(profile.bin_centers)
        self.n_time = len(self.time_array)
        self.R = np.asarray(resonators.R_S, dtype=np.float64)
        self.omega_r = omega_R
        self.Q = Q
        self.n_resonators = len(self.R)
        self._Qtilde = self.Q * np.sqrt(1.0 - 1.0 / (4.0 * self.Q ** 2.0))
        self._reOmegaP = self.omega_r * self._Qtilde / self.Q
        self._imOmegaP = self.omega_r / (2.0 * self.Q)
        self._time_dev = torch.as_tensor(np.asarray(
            self.time_array.cpu() if isinstance(self.time_array, torch.Tensor)
            else self.time_array, dtype=np.float64), device="cuda")
        wake_length = len(self.time_array) * profile.bin_size
        _InducedVoltage.__init__(self, beam, profile, frequency_resolution=None,
                                 wake_length=wake_length,
                                 multi_turn_wake=multi_turn_wake,
                                 rf_station=rf_station, mtw_mode="time",
                                 use_regular_fft=True)

    def process(self):
        """impedance.py:1263-1284: sizes follow the (re)sliced profile."""
        _InducedVoltage.process(self)
        S = int(self.profile.n_slices)
        self._bc_dev = torch.as_tensor(np.asarray(self.profile.bin_centers,
                                                  dtype=np.float64), device="cuda")
        step = _RESONATORS_PER_LAUNCH
        groups = [(i, min(i + step, self.n_resonators))
                  for i in range(0, self.n_resonators, step)]
        self._groups = groups
        self._workspace = bm.resonator_workspace(S, groups[0][1] - groups[0][0])
        off = (groups[0][1] - groups[0][0]) * S * 16
        # kappa_k of the last evaluation, a view into the kernel's scratch
        self._kappa1 = self._workspace[off: off + 8 * (S - 1)].view(torch.float64)
        self._deltaT = None
        self._tmp_matrix = torch.ones((self.n_resonators, self.n_time),
                                      dtype=torch.float64, device="cuda")
        self.induced_voltage = torch.zeros(self.n_time,
                                           dtype=self.profile.n_macroparticles.dtype,
                                           device="cuda")

    def induced_voltage_1turn(self, beam_spectrum_dict=None):
        """impedance.py:1286-1315."""
        scale = -self.beam.particle.charge * e * self.beam.n_macroparticles \
            * self.beam.ratio
        total = None
        for lo, hi in self._groups:
            v, _ = bm.resonator_induced_voltage(
                self.profile.n_macroparticles, self._bc_dev, self.profile.bin_size,
                self.beam.n_macroparticles, self._time_dev, self.R[lo:hi],
                self.omega_r[lo:hi], self.Q[lo:hi], 1.0 if len(self._groups) > 1 else scale,
                tmp_matrix=self._tmp_matrix[lo:hi], workspace=self._workspace)
            total = v if total is None else total + v
        if len(self._groups) > 1:
            total = total * scale
        self.induced_voltage = total.to(self.profile.n_macroparticles.dtype)

    def induced_voltage_mtw(self, beam_spectrum_dict=None):
        """impedance.py:1317-1335: drop one window of memory, add this
        turn's voltage at the first n_time points, read those back.  In
        double precision with at most 64 modes this is one fused launch
        pair writing a new memory tensor (blond_resonator_mtw_f64)."""
        S = int(self.array_length)
        n_t = int(self.n_time)
        mem = self.mtw_memory
        if mem.dtype == torch.float64 and len(self._groups) == 1:
            scale = -self.beam.particle.charge * e * self.beam.n_macroparticles \
                * self.beam.ratio
            self.mtw_memory, _ = bm.resonator_induced_voltage(
                self.profile.n_macroparticles, self._bc_dev, self.profile.bin_size,
                self.beam.n_macroparticles, self._time_dev, self.R, self.omega_r,
                self.Q, scale, tmp_matrix=self._tmp_matrix, workspace=self._workspace,
                memory_in=mem, shift=S)
        else:
            self.mtw_memory = torch.cat((mem, mem.new_zeros(S)))[S:].contiguous()
            self.induced_voltage_1turn(beam_spectrum_dict)
            self.mtw_memory[:n_t] += self.induced_voltage.to(self.mtw_memory.dtype)
        self.induced_voltage = self.mtw_memory[:n_t]
