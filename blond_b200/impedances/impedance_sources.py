"""Resonator impedance source (blond/impedances/impedance_sources.py:239-471)."""
from __future__ import annotations

import numpy as np

from .. import bmath as bm


class Resonators:
    """Z(f) = R / (1 + jQ (f/f_r - f_r/f)), summed over the modes."""

    def __init__(self, R_S, frequency_R, Q):
        self.R_S = np.array([R_S], dtype=float).flatten()
        self.frequency_R = np.array([frequency_R], dtype=float).flatten()
        self.Q = np.array([Q], dtype=float).flatten()
        if np.count_nonzero(self.Q < 0.5) > 0:
            raise RuntimeError("All quality factors Q must be greater or equal 0.5")
        self.n_resonators = len(self.R_S)
        self.impedance = 0
        self.wake = None

    @property
    def frequency_R(self):
        return self._frequency_R

    @frequency_R.setter
    def frequency_R(self, f):
        self._frequency_R = np.asarray(f, dtype=float)
        self._omega_R = 2 * np.pi * self._frequency_R

    @property
    def omega_R(self):
        return self._omega_R

    def imped_calc(self, frequency_array):
        """impedance_sources.py:382-414 via the fast_resonator kernel
        (cpp_routines/fast_resonator.cpp:19-74); complex128 device tensor."""
        self.frequency_array = frequency_array
        self.impedance = bm.fast_resonator(self.R_S, self.Q, frequency_array,
                                           self.frequency_R)

    def wake_calc(self, time_array):
        """impedance_sources.py:345-380 (setup-time, host)."""
        t = np.asarray(time_array, dtype=float)
        self.time_array = t
        self.wake = np.zeros(t.shape)
        for i in range(self.n_resonators):
            alpha = self.omega_R[i] / (2 * self.Q[i])
            omega_bar = np.sqrt(self.omega_R[i] ** 2 - alpha**2)
            self.wake += ((np.sign(t) + 1) * self.R_S[i] * alpha * np.exp(-alpha * t)
                          * (np.cos(omega_bar * t)
                             - alpha / omega_bar * np.sin(omega_bar * t)))
