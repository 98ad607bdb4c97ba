"""Profile slicing (blond/beam/profile.py:44-991), hot path on the B200.

``Profile.track()`` runs ``slice_beam`` (or ``slice_smooth``) over the
device coordinates into ``n_macroparticles``, a device tensor in the beam's
precision.  Edges and bin centres are computed on the host exactly as the
reference does (np.linspace, then midpoints) and kept both as numpy arrays
and as device tensors (``bin_centers_dev``).
"""
from __future__ import annotations

import numpy as np
import torch

from .. import bmath as bm


class CutOptions:
    """Slicing frame (profile.py:44-259)."""

    def __init__(self, cut_left=None, cut_right=None, n_slices: int = 100,
                 n_sigma=None, cuts_unit: str = "s", rf_station=None):
        self.cut_left = float(cut_left) if cut_left is not None else None
        self.cut_right = float(cut_right) if cut_right is not None else None
        self.n_slices = int(n_slices)
        self.n_sigma = float(n_sigma) if n_sigma is not None else None
        self.cuts_unit = cuts_unit
        self.rf_station = rf_station
        if cuts_unit == "rad" and rf_station is None:
            raise RuntimeError('Argument "rf_station" required to convert from '
                               "radians to seconds")
        if cuts_unit not in ("rad", "s"):
            raise NameError(f'cuts_unit should be "s" or "rad", not {cuts_unit=} !')
        self.edges = np.zeros(self.n_slices + 1)
        self.bin_centers = np.zeros(self.n_slices)
        self.bin_size = 0.0

    def set_cuts(self, beam=None):
        """profile.py:175-211."""
        if self.cut_left is None and self.cut_right is None:
            # one device reduction (blond_cut_limits): min/max -/+ 5 % of the
            # spread, or mean -/+ n_sigma sigma / 2; read back once
            cuts = bm.cut_limits(beam.dt, self.n_sigma).cpu().numpy()
            self.cut_left, self.cut_right = float(cuts[0]), float(cuts[1])
        else:
            self.cut_left = float(self.convert_coordinates(self.cut_left, self.cuts_unit))
            self.cut_right = float(self.convert_coordinates(self.cut_right, self.cuts_unit))
        self.edges = np.linspace(self.cut_left, self.cut_right,
                                 self.n_slices + 1).astype(bm.precision.real_t)
        self.bin_centers = (self.edges[:-1] + self.edges[1:]) / 2
        self.bin_size = (self.cut_right - self.cut_left) / self.n_slices

    def convert_coordinates(self, value: float, input_unit_type: str) -> float:
        if input_unit_type == "s":
            return value
        if input_unit_type == "rad":
            return value / float(self.rf_station.omega_rf[0, self.rf_station.counter[0]])
        raise NameError(input_unit_type)

    def get_slices_parameters(self):
        return (self.n_slices, self.cut_left, self.cut_right, self.n_sigma,
                self.edges, self.bin_centers, self.bin_size)


class FitOptions:
    def __init__(self, fit_option=None, fit_extra_options=None):
        self.fit_option = fit_option
        self.fit_extra_options = fit_extra_options


class FilterOptions:
    def __init__(self, filter_method=None, filter_extra_options=None):
        self.filter_method = filter_method
        self.filter_extra_options = filter_extra_options


class OtherSlicesOptions:
    def __init__(self, smooth: bool = False, direct_slicing: bool = True):
        self.smooth = smooth
        self.direct_slicing = direct_slicing


class Profile:
    """Beam profile on the device (profile.py:561-719)."""

    def __init__(self, beam, cut_options: CutOptions | None = None,
                 fit_options: FitOptions | None = None,
                 filter_options: FilterOptions | None = None,
                 other_slices_options: OtherSlicesOptions | None = None):
        cut_options = cut_options or CutOptions()
        fit_options = fit_options or FitOptions()
        filter_options = filter_options or FilterOptions()
        other_slices_options = other_slices_options or OtherSlicesOptions()
        if filter_options.filter_method is not None:
            raise NotImplementedError(
                "profile filters are host-side diagnostics outside the tracking "
                "hot path; use the reference toolbox on a host copy")
        self.cut_options = cut_options
        cut_options.set_cuts(beam)
        self.beam = beam
        (self.n_slices, self.cut_left, self.cut_right, self.n_sigma, self.edges,
         self.bin_centers, self.bin_size) = cut_options.get_slices_parameters()
        dtype = beam.dt.dtype if beam is not None else bm.precision.torch_t
        self.bin_centers_dev = torch.as_tensor(self.bin_centers, device="cuda").to(dtype)
        self.n_macroparticles = torch.zeros(self.n_slices, dtype=dtype, device="cuda")
        self.beam_spectrum = None
        self.beam_spectrum_freq = np.array([])
        self.smooth = bool(other_slices_options.smooth)
        self.operations = [self._slice_smooth if self.smooth else self._slice]
        self.fit_option = fit_options.fit_option
        self.fit_extra_options = None
        if self.fit_option is not None:
            self.bunchPosition = 0.0
            self.bunchLength = 0.0
            fits = {"gaussian": self.apply_fit, "rms": self.rms, "fwhm": self.fwhm}
            if self.fit_option not in fits:
                raise NameError(f"{fit_options=}")
            self.operations.append(fits[self.fit_option])
        if other_slices_options.direct_slicing and beam is not None:
            self.track()

    def track(self):
        for op in self.operations:
            op()

    def _slice(self):
        bm.slice_beam(self.beam.dt, self.n_macroparticles, self.cut_left,
                      self.cut_right)

    def _slice_smooth(self):
        bm.slice_smooth(self.beam.dt, self.n_macroparticles, self.cut_left,
                        self.cut_right)

    # ------------------------------------------------------------ fits
    # Bunch position and length (4 sigma) after each slicing, as the
    # reference's Profile.apply_fit / rms / fwhm (profile.py:775-866) with
    # toolbox/filters_and_fitting.py:129-215.  They are per-turn
    # diagnostics, not part of the tracking arithmetic: rms reduces on the
    # device; the Gaussian least-squares fit and the FWHM edge search run on
    # a host copy of the profile, as the reference's GPU backend does for
    # the fit (filters_and_fitting.py:138-141).
    def apply_fit(self):
        from scipy.optimize import curve_fit
        y = self.n_macroparticles.double().cpu().numpy()
        x = np.asarray(self.bin_centers, dtype=np.float64)
        if self.bunchLength == 0:
            dt = self.beam.dt.double()
            p0 = [float(y.max()), float(dt.mean()), float(dt.std(unbiased=False))]
        else:
            p0 = [float(y.max()), float(self.bunchPosition), float(self.bunchLength / 4.0)]
        self.fit_extra_options = curve_fit(_gauss, x, y, p0)[0]
        self.bunchPosition = self.fit_extra_options[1]
        self.bunchLength = 4 * self.fit_extra_options[2]

    def rms(self):
        y = self.n_macroparticles.double()
        x = torch.as_tensor(np.asarray(self.bin_centers, dtype=np.float64), device=y.device)
        dx = float(self.bin_centers[1] - self.bin_centers[0])
        line = y / torch.trapezoid(y, dx=dx)
        bp = torch.trapezoid(x * line, dx=dx)
        bl = 4 * torch.sqrt(torch.trapezoid((x - bp) ** 2 * line, dx=dx))
        self.bunchPosition, self.bunchLength = float(bp), float(bl)

    def fwhm(self, shift: float = 0):
        y = self.n_macroparticles.double().cpu().numpy()
        x = np.asarray(self.bin_centers, dtype=np.float64)
        self.bunchPosition, self.bunchLength = _fwhm(y, x, shift)

    def beam_spectrum_freq_generation(self, n_sampling_fft: int):
        self.beam_spectrum_freq = bm.rfftfreq(n_sampling_fft, self.bin_size)

    def beam_spectrum_generation(self, n_sampling_fft: int):
        self.beam_spectrum = bm.rfft(self.n_macroparticles, n_sampling_fft)

    def beam_profile_derivative(self, mode: str = "gradient"):
        """profile.py:905-937 ('gradient' only): np.gradient on the device."""
        if mode != "gradient":
            raise NotImplementedError(f"derivative mode {mode!r}")
        dist = float(self.bin_centers[1] - self.bin_centers[0])
        p = self.n_macroparticles.double()
        d = torch.empty_like(p)
        d[1:-1] = (p[2:] - p[:-2]) / (2.0 * dist)
        d[0] = (p[1] - p[0]) / dist
        d[-1] = (p[-1] - p[-2]) / dist
        return self.bin_centers, d


def _gauss(x, *p):
    """A exp(-(x - x0)^2 / (2 sx^2)) (filters_and_fitting.py:146-155)."""
    A, x0, sx = p
    return A * np.exp(-((x - x0) ** 2) / 2.0 / sx ** 2)


def _fwhm(y, x, shift=0.0):
    """Bunch position and 4-sigma length from the full width at half
    maximum with linear interpolation of both edges
    (filters_and_fitting.py:179-211); (nan, nan) when the right edge is the
    last bin (at the first bin the left neighbour wraps to the last, as
    numpy indexing does in the reference)."""
    half = shift + 0.5 * (y.max() - shift)
    above = np.where(y >= half)[0]
    t1, t2 = above[0], above[-1]
    w = x[1] - x[0]
    try:
        t_left = x[t1] - w * (y[t1] - half) / (y[t1] - y[t1 - 1])
        t_right = x[t2] + w * (y[t2] - half) / (y[t2] - y[t2 + 1])
    except IndexError:
        return np.nan, np.nan
    return (t_left + t_right) / 2, 4 * (t_right - t_left) / (2 * np.sqrt(2 * np.log(2)))
