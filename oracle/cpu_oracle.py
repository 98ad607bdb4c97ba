"""ORACLE -- test infrastructure, not product code.

Python face of the CPU oracle: ctypes bindings of oracle/_build/liboracle.so
(the plain-C restatement in blond_oracle.c) plus the reference's FFT step
restated with numpy.fft (pocketfft, numpy 2.3 -- the library the reference
itself calls, blond/utils/bmath_backends.py:447-449), and a multi-turn
driver in the reference main-loop order
[TotalInducedVoltage.track, RingAndRFTracker.track, Profile.track]
(__EXAMPLES/main_files/EX_05_Wake_impedance.py:318-339).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this module, and only as a checker or a timed CPU baseline.
"""
from __future__ import annotations

import ctypes as ct
import os
import subprocess

import numpy as np
from scipy.constants import e as E_CHARGE

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
_lib = None


def load() -> ct.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
        _lib = ct.CDLL(LIB)
    return _lib


def _P(a: np.ndarray):
    return a.ctypes.data_as(ct.c_void_p)


def _r(dtype):
    return ct.c_double if dtype == np.float64 else ct.c_float


def _suf(dtype):
    return "f64" if dtype == np.float64 else "f32"


def kick(dt, dE, voltage, omega, phi, charge, acc):
    """In place on dE (kick.cpp:16-35)."""
    lib, r, t = load(), _r(dt.dtype), dt.dtype
    V, om, ph = (np.ascontiguousarray(x, dtype=t) for x in (voltage, omega, phi))
    getattr(lib, f"oracle_kick_{_suf(t)}")(
        _P(dt), _P(dE), ct.c_int(len(V)), r(charge), _P(V), _P(om), _P(ph),
        ct.c_int(len(dt)), r(acc))


def rf_volt_comp(voltage, omega, phi, bin_centers):
    lib = load()
    t = bin_centers.dtype
    out = np.zeros(len(bin_centers), dtype=t)
    V, om, ph = (np.ascontiguousarray(x, dtype=t) for x in (voltage, omega, phi))
    getattr(lib, f"oracle_rf_volt_comp_{_suf(t)}")(
        _P(V), _P(om), _P(ph), _P(bin_centers), ct.c_int(len(V)),
        ct.c_int(len(bin_centers)), _P(out))
    return out


def drift(dt, dE, solver, t_rev, length_ratio, alpha_order, eta_0, eta_1,
          eta_2, alpha_0, alpha_1, alpha_2, beta, energy):
    """In place on dt (drift.cpp:19-78); solver 0/1/2."""
    lib, r = load(), _r(dt.dtype)
    getattr(lib, f"oracle_drift_{_suf(dt.dtype)}")(
        _P(dt), _P(dE), ct.c_int(solver), r(t_rev), r(length_ratio),
        r(alpha_order), r(eta_0), r(eta_1), r(eta_2), r(alpha_0), r(alpha_1),
        r(alpha_2), r(beta), r(energy), ct.c_int(len(dt)))


def histogram(dt, cut_left, cut_right, n_slices):
    """histogram.cpp:22-73; returns a new array of dt's dtype."""
    lib, r = load(), _r(dt.dtype)
    out = np.zeros(n_slices, dtype=dt.dtype)
    getattr(lib, f"oracle_histogram_{_suf(dt.dtype)}")(
        _P(dt), _P(out), r(cut_left), r(cut_right), ct.c_int(n_slices),
        ct.c_int(len(dt)))
    return out


def smooth_histogram(dt, cut_left, cut_right, n_slices):
    lib, r = load(), _r(dt.dtype)
    out = np.zeros(n_slices, dtype=dt.dtype)
    getattr(lib, f"oracle_smooth_histogram_{_suf(dt.dtype)}")(
        _P(dt), _P(out), r(cut_left), r(cut_right), ct.c_int(n_slices),
        ct.c_int(len(dt)))
    return out


def linear_interp_kick(dt, dE, voltage, bin_centers, charge, acc):
    lib, r, t = load(), _r(dt.dtype), dt.dtype
    V = np.ascontiguousarray(voltage, dtype=t)
    bc = np.ascontiguousarray(bin_centers, dtype=t)
    getattr(lib, f"oracle_linear_interp_kick_{_suf(t)}")(
        _P(dt), _P(dE), _P(V), _P(bc), r(charge), ct.c_int(len(bc)),
        ct.c_int(len(dt)), r(acc))


def fast_resonator(R, Q, freq, fr):
    lib = load()
    f = np.ascontiguousarray(freq, dtype=np.float64)
    re = np.zeros(len(f))
    im = np.zeros(len(f))
    R, Q, fr = (np.ascontiguousarray(x, dtype=np.float64) for x in (R, Q, fr))
    lib.oracle_fast_resonator_f64(_P(re), _P(im), _P(f), _P(R), _P(Q), _P(fr),
                                  ct.c_int(len(R)), ct.c_int(len(f)))
    return re + 1j * im


def beam_phase(bin_centers, profile, alpha, omega_rf, phi_rf, bin_size, weighted=True):
    """beam_phase.cpp:6-65 (weighted) / beam_phase_fast (weighted=False)."""
    lib = load()
    bc = np.ascontiguousarray(bin_centers)
    p = np.ascontiguousarray(profile, dtype=bc.dtype)
    r = _r(bc.dtype)
    f = getattr(lib, f"oracle_beam_phase_{_suf(bc.dtype)}")
    f.restype = r
    return float(f(_P(bc), _P(p), r(alpha), r(omega_rf), r(phi_rf), r(bin_size),
                   ct.c_int(len(bc)), ct.c_int(1 if weighted else 0)))


def induced_voltage(profile, total_impedance, n_fft, charge, ratio, n_out):
    """impedance.py:475-489 with numpy.fft."""
    spec = np.fft.rfft(profile, n_fft)
    v = -(charge * E_CHARGE * ratio * np.fft.irfft(total_impedance * spec))
    return v[:n_out]


def track_oracle(dt0, dE0, ring, rf, cuts, bin_centers, n_slices, n_turns,
                 impedance=None, intensity=1e10, solver=0, inductive=None,
                 start_turn=0):
    """Multi-turn CPU tracking in the reference main-loop order.

    impedance = (n_fft, total_impedance) for the FFT induced voltage;
    inductive = Z_over_n per turn (InductiveImpedance, 'gradient').
    Returns (dt, dE, profiles[n_turns+1], induced_voltages[n_turns]).
    """
    dt = np.array(dt0, dtype=np.float64)
    dE = np.array(dE0, dtype=np.float64)
    q = float(rf.particle.charge)
    ratio = intensity / len(dt)
    cl, cr = cuts
    bc = np.asarray(bin_centers, dtype=np.float64)
    prof = histogram(dt, cl, cr, n_slices)
    profiles, vinds = [prof], []
    bin_size = (cr - cl) / n_slices
    for k in range(n_turns):
        t = start_turn + k
        if impedance is not None:
            n_fft, Z = impedance
            v = induced_voltage(prof, Z, n_fft, q, ratio, n_slices)
            if inductive is not None:
                deriv = np.gradient(prof, bc[1] - bc[0])
                v = v + -(q * E_CHARGE / (2 * np.pi) * ratio * inductive[t]
                          * rf.t_rev[t] / bin_size * deriv)
            vinds.append(v)
            linear_interp_kick(dt, dE, v, bc, q, 0.0)
        kick(dt, dE, rf.voltage[:, t], rf.omega_rf[:, t], rf.phi_rf[:, t], q,
             -rf.delta_E[t])
        drift(dt, dE, solver, rf.t_rev[t + 1], rf.length_ratio, rf.alpha_order,
              rf.eta_0[t + 1], rf.eta_1[t + 1], rf.eta_2[t + 1],
              rf.alpha_0[t + 1], rf.alpha_1[t + 1], rf.alpha_2[t + 1],
              rf.beta[t + 1], rf.energy[t + 1])
        prof = histogram(dt, cl, cr, n_slices)
        profiles.append(prof)
    return dt, dE, np.array(profiles), vinds


def track_oracle_fixed(dt0, q0, unit, ring, rf, cuts, bin_centers, n_slices, n_turns,
                       impedance=None, intensity=1e10, start_turn=0):
    """The fixed-point energy form (dE = q * unit, q an int32 count) on the
    CPU, in the reference main-loop order: each turn's energy change -- the
    induced-voltage kick (linear_interp_kick.cpp:21-71) then the RF kick
    (kick.cpp:16-35), evaluated by the same routines on a zero energy
    array, i.e. in float64 and in the reference's order -- is rounded once
    to a whole number of units; the simple drift (drift.cpp:19-28) then
    uses q * unit.  Returns (dt, q, profiles[n_turns+1]).
    """
    dt = np.array(dt0, dtype=np.float64)
    q = np.array(q0, dtype=np.int64)
    qc = float(rf.particle.charge)
    ratio = intensity / len(dt)
    cl, cr = cuts
    bc = np.asarray(bin_centers, dtype=np.float64)
    prof = histogram(dt, cl, cr, n_slices)
    profiles = [prof]
    for k in range(n_turns):
        t = start_turn + k
        inc = np.zeros_like(dt)
        if impedance is not None:
            n_fft, Z = impedance
            v = induced_voltage(prof, Z, n_fft, qc, ratio, n_slices)
            linear_interp_kick(dt, inc, v, bc, qc, 0.0)
        kick(dt, inc, rf.voltage[:, t], rf.omega_rf[:, t], rf.phi_rf[:, t], qc,
             -rf.delta_E[t])
        q = q + np.rint(inc * (1.0 / unit)).astype(np.int64)
        if np.abs(q).max() > 2**31 - 1:
            raise OverflowError("energy beyond the 32-bit grid")
        dE = q.astype(np.float64) * unit
        drift(dt, dE, 0, rf.t_rev[t + 1], rf.length_ratio, rf.alpha_order,
              rf.eta_0[t + 1], rf.eta_1[t + 1], rf.eta_2[t + 1],
              rf.alpha_0[t + 1], rf.alpha_1[t + 1], rf.alpha_2[t + 1],
              rf.beta[t + 1], rf.energy[t + 1])
        prof = histogram(dt, cl, cr, n_slices)
        profiles.append(prof)
    return dt, q, np.array(profiles)
