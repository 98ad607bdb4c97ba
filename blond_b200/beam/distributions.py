"""Bunch generation (blond/beam/distributions.py:1194-1278, 1367-1430).

The random streams are the reference's (numpy default_rng(seed) for dt and
default_rng(seed + 1) for dE), drawn on the host so that a given seed gives
the same macro-particles as the reference, then uploaded once.
"""
from __future__ import annotations

import warnings

import numpy as np
import torch


def _get_dE_from_dt(ring, rf_station, dt_amplitude: float) -> float:
    """Single-harmonic Hamiltonian dE amplitude (distributions.py:1367-1430)."""
    if rf_station.n_rf > 1:
        warnings.warn("bigaussian(): only the first RF harmonic is used to "
                      "match sigma_dE")
    t = rf_station.counter[0]
    harmonic = rf_station.harmonic[0, t]
    energy = rf_station.energy[t]
    beta = rf_station.beta[t]
    omega_rf = rf_station.omega_rf[0, t]
    phi_s = rf_station.phi_s[t]
    eta0 = rf_station.eta_0[t]
    voltage = rf_station.charge * rf_station.voltage[0, t]
    phi_b = omega_rf * dt_amplitude + phi_s
    return np.sqrt(voltage * energy * beta**2
                   * (np.cos(phi_b) - np.cos(phi_s) + (phi_b - phi_s) * np.sin(phi_s))
                   / (np.pi * harmonic * np.fabs(eta0)))


def bigaussian_arrays(n: int, sigma_dt: float, sigma_dE: float, centre: float,
                      seed: int):
    """Host float64 coordinates of the reference's streams
    (distributions.py:1241-1256)."""
    rng_dt = np.random.default_rng(seed)
    rng_dE = np.random.default_rng(seed + 1)
    dt = sigma_dt * rng_dt.normal(size=n) + centre
    dE = sigma_dE * rng_dE.normal(size=n)
    return dt, dE


def bigaussian(ring, rf_station, beam, sigma_dt: float, sigma_dE=None,
               seed: int = 1234, reinsertion: bool = False):
    """Fill beam.dt / beam.dE with a bi-Gaussian bunch centred in the bucket."""
    if reinsertion:
        raise NotImplementedError("bigaussian(reinsertion=True) is not supported")
    if sigma_dE is None:
        sigma_dE = _get_dE_from_dt(ring, rf_station, sigma_dt)
    t = rf_station.counter[0]
    omega_rf = rf_station.omega_rf[0, t]
    phi_s = rf_station.phi_s[t]
    phi_rf = rf_station.phi_rf[0, t]
    if rf_station.eta_0[t] < 0:
        phi_rf -= np.pi
    beam.sigma_dt = sigma_dt
    beam.sigma_dE = sigma_dE
    dt, dE = bigaussian_arrays(beam.n_macroparticles, sigma_dt, sigma_dE,
                               (phi_s - phi_rf) / omega_rf, seed)
    dtype = beam.dt.dtype
    dev = beam.dt.device
    beam.dt = torch.from_numpy(dt).to(device=dev, dtype=dtype)
    beam.dE = torch.from_numpy(dE).to(device=dev, dtype=beam.dE.dtype)
