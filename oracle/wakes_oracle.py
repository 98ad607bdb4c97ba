"""CPU restatement of the time-domain wake arithmetic (test infrastructure).

The checker for blond_b200/csrc/wakes.cu and the multi-turn-wake objects of
blond_b200/impedances/impedance.py.  Only tests import it.

* resonator_induced_voltage: the reference's analytic resonator
  convolution evaluated the reference's way, as the full time x bin
  matrix (blond/utils/butils_wrap_python.py:656-790, called by
  InducedVoltageResonator.induced_voltage_1turn,
  blond/impedances/impedance.py:1286-1315).
* resonator_mtw: InducedVoltageResonator's multi-turn memory over turns
  (impedance.py:1317-1335).
* shift_trev_time: the 'time' multi-turn-wake memory shift
  (impedance.py:533-550), which is numpy.interp.

Pinned against the reference's own outputs stored in
tests/golden/wakes_resonator.npz and mtw_resonator.npz
(tests/golden/gen_golden.py).
"""
from __future__ import annotations

import numpy as np
from scipy.constants import e as E_CHARGE


def resonator_constants(omega_r, Q):
    """(Qtilde, a, b) with Qtilde = Q sqrt(1 - 1/(4 Q^2)), a = omega Qtilde
    / Q, b = omega / (2 Q) (impedance.py:1218-1220)."""
    omega_r = np.asarray(omega_r, dtype=np.float64)
    Q = np.asarray(Q, dtype=np.float64)
    qt = Q * np.sqrt(1.0 - 1.0 / (4.0 * Q ** 2.0))
    return qt, omega_r * qt / Q, omega_r / (2.0 * Q)


def resonator_wake_step(D, a, b, qt):
    """F(D) = (2 cos(a D) + sin(a D) / qt) exp(-b D) H(D) - sign(D) with the
    Heaviside H(D) = (sign(D) + 1) / 2 (butils_wrap_python.py:764-777)."""
    with np.errstate(over="ignore", invalid="ignore"):
        osc = (2 * np.cos(a * D) + np.sin(a * D) / qt) * np.exp(-b * D)
        return osc * 0.5 * (np.sign(D) + 1) - np.sign(D)


def resonator_induced_voltage(profile, bin_centers, bin_size, n_macroparticles,
                              time_array, R, omega_r, Q, charge=1.0, ratio=1.0,
                              per_resonator=False):
    """V(t_j) = -charge e N ratio sum_r R_r / (2 w_r Q_r)
    sum_k kappa_k (F_r(t_j - bc_{k+1}) - F_r(t_j - bc_k)),
    kappa = diff(profile) / diff(bc) / (N bin_size)
    (butils_wrap_python.py:756-790).  Row blocks of the time x bin matrix
    keep the memory bounded."""
    prof = np.asarray(profile, dtype=np.float64)
    bc = np.asarray(bin_centers, dtype=np.float64)
    t = np.asarray(time_array, dtype=np.float64)
    R = np.asarray(R, dtype=np.float64).reshape(-1)
    kappa = np.diff(prof) / np.diff(bc) / (n_macroparticles * bin_size)
    qt, a, b = resonator_constants(omega_r, Q)
    omega_r = np.asarray(omega_r, dtype=np.float64).reshape(-1)
    Q = np.asarray(Q, dtype=np.float64).reshape(-1)
    rows = np.zeros((len(R), len(t)))
    block = max(1, (1 << 22) // max(1, len(bc)))
    for j0 in range(0, len(t), block):
        D = t[j0:j0 + block, None] - bc[None, :]
        for r in range(len(R)):
            F = resonator_wake_step(D, a[r], b[r], qt[r])
            rows[r, j0:j0 + block] = (R[r] / (2 * omega_r[r] * Q[r])
                                      * np.sum(kappa * np.diff(F), axis=1))
    v = rows.sum(axis=0) * (-charge * E_CHARGE * n_macroparticles * ratio)
    return (v, rows) if per_resonator else v


def resonator_mtw(memory, voltage, n_window):
    """One turn of InducedVoltageResonator's memory (impedance.py:1317-1335):
    drop the first n_window points, pad zeros, add this turn's voltage at
    the front; returns (memory, induced_voltage)."""
    mem = np.append(np.asarray(memory, dtype=np.float64), np.zeros(n_window))[n_window:]
    n_t = len(voltage)
    mem[:n_t] += voltage
    return mem, mem[:n_t].copy()


def shift_trev_time(memory, time_mtw, t_rev):
    """impedance.py:533-550: memory(t + t_rev) on time_mtw, 0 outside."""
    return np.interp(time_mtw + t_rev, time_mtw, memory, left=0, right=0)
