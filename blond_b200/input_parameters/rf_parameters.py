"""RFStation: per-turn RF programme (blond/input_parameters/rf_parameters.py:239-446).

Host-side parameter source.  Programmes are [n_rf, n_turns+1] arrays in
Fortran order so that one turn's column is contiguous, as in the reference;
the tracker uploads them to the device once.
"""
from __future__ import annotations

import numpy as np
from scipy.constants import c


def _rf_array(x, n_rf: int, n_turns: int, name: str) -> np.ndarray:
    a = np.asarray(x, dtype=float)
    if a.ndim == 0:
        a = a.reshape(1)
    if a.ndim == 1:
        if a.size == n_rf:
            return np.tile(a.reshape(n_rf, 1), (1, n_turns + 1))
        if n_rf == 1 and a.size == n_turns + 1:
            return a.reshape(1, -1).copy()
    if a.ndim == 2 and a.shape == (n_rf, n_turns + 1):
        return a.copy()
    raise NotImplementedError(
        f"{name}: give one value per RF system or an [n_rf, n_turns+1] "
        "array; time-interpolated programmes are not supported")


class RFStation:
    def __init__(self, ring, harmonic, voltage, phi_rf_d, n_rf: int = 1,
                 section_index: int = 1, omega_rf=None, phi_noise=None,
                 phi_modulation=None, rf_station_options=None):
        if phi_modulation is not None:
            raise NotImplementedError("phi_modulation is not supported")
        self.counter = [int(0)]
        self.section_index = int(section_index - 1)
        self.n_rf = int(n_rf)
        self.particle = ring.particle
        self.n_turns = ring.n_turns
        self.ring_circumference = ring.ring_circumference
        self.section_length = ring.ring_length[self.section_index]
        self.length_ratio = float(self.section_length / self.ring_circumference)
        self.t_rev = ring.t_rev
        s = self.section_index
        self.momentum = ring.momentum[s]
        self.beta = ring.beta[s]
        self.gamma = ring.gamma[s]
        self.energy = ring.energy[s]
        self.delta_E = ring.delta_E[s]
        self.alpha_order = ring.alpha_order
        self.charge = self.particle.charge
        for i in range(3):
            setattr(self, f"alpha_{i}", getattr(ring, f"alpha_{i}")[s])
            setattr(self, f"eta_{i}", getattr(ring, f"eta_{i}")[s])
        self.sign_eta_0 = np.sign(self.eta_0)
        nt = self.n_turns
        self.harmonic = _rf_array(harmonic, self.n_rf, nt, "harmonic")
        self.voltage = np.asfortranarray(_rf_array(voltage, self.n_rf, nt, "voltage"))
        self.empty = bool(np.sum(self.voltage) == 0)
        self.phi_rf_d = _rf_array(phi_rf_d, self.n_rf, nt, "phi_rf_d")
        if omega_rf is None:
            self.omega_rf_d = (2.0 * np.pi * self.beta * c * self.harmonic
                               / self.ring_circumference)
        else:
            self.omega_rf_d = _rf_array(omega_rf, self.n_rf, nt, "omega_rf")
        self.phi_noise = None if phi_noise is None else \
            _rf_array(phi_noise, self.n_rf, nt, "phi_noise")
        self.phi_modulation = None
        self.phi_rf = np.array(self.phi_rf_d, order="F", dtype=float)
        self.dphi_rf = np.zeros(self.n_rf)
        self.omega_rf = np.array(self.omega_rf_d, order="F", dtype=float)
        self.t_rf = 2 * np.pi / self.omega_rf
        if not self.empty:
            self.phi_s = calculate_phi_s(self, self.particle)
            self.Q_s = calculate_Q_s(self, self.particle)
            self.omega_s0 = self.Q_s * ring.omega_rev


def calculate_Q_s(rf_station, particle):
    """rf_parameters.py:610-636 (single harmonic, no intensity effects)."""
    return np.sqrt(rf_station.harmonic[0] * np.abs(particle.charge)
                   * rf_station.voltage[0]
                   * np.abs(rf_station.eta_0 * np.cos(rf_station.phi_s))
                   / (2 * np.pi * rf_station.beta**2 * rf_station.energy))


def calculate_phi_s(rf_station, particle, accelerating_systems: str = "as_single"):
    """rf_parameters.py:640-721, the default 'as_single' branch."""
    if accelerating_systems != "as_single":
        raise NotImplementedError(accelerating_systems)
    eta0 = rf_station.eta_0
    denergy = np.append(rf_station.delta_E, rf_station.delta_E[-1])
    ratio = denergy / (particle.charge * rf_station.voltage[0, :])
    phi_s = np.arcsin(ratio)
    mid = np.append((eta0[1:] + eta0[:-1]) / 2, eta0[-1])
    above = np.where(mid > 0)[0]
    below = np.where(mid < 0)[0]
    h = np.heaviside(np.sign(particle.charge), 0) * np.pi
    phi_s[above] = (h - phi_s[above]) % (2 * np.pi)
    phi_s[below] = (h + phi_s[below]) % (2 * np.pi)
    return phi_s
