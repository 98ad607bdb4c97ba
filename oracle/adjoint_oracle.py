"""CPU restatement of the differentiable N-turn map (test infrastructure).

This is the checker for blond_b200/adjoint.py and its kernels: numpy FP64,
vectorised per turn, for small particle counts.  Only tests import it.

The map follows the reference main loop's order per turn
(blond/impedances/impedance.py:113-146, :457-489 for the induced voltage
with numpy's FFT; blond/trackers/tracker.py:521-615 for kick then drift;
blond/cpp_routines/kick.cpp:16-35, drift.cpp:19-40 'simple'), with two
stated differences from the reference's own functions, both needed for a
derivative to exist or be accurate:

* the profile is cloud-in-cell on the bin centres (the reference's
  smooth_histogram, histogram.cpp:75-132, jumps by whole particles);
* the interpolated kick is q (V_k (1-u) + V_k+1 u), the same function as
  linear_interp_kick.cpp:44-62 without its slope/offset cancellation.

Parity of this restatement with the reference is pinned where the two
coincide: with the induced voltage off, kick and drift are the reference's
formulas, and tests compare them with the reference-pinned oracle
(oracle/cpu_oracle.py) on the same inputs.
"""
from __future__ import annotations

import numpy as np
from scipy.constants import e as E_CHARGE


def fixed_bits(n):
    """Fixed-point bits per particle of the deposit: min(52, 62 -
    ceil(log2(n + 1))), so n particles' units stay below 2^63."""
    return min(52, 62 - int(np.ceil(np.log2(n + 1))) if n > 0 else 52)


def cic(dt, n_slices, bc0, inv_w):
    """Cloud-in-cell profile: bin floor(f) gets 1-u, the next bin u, with
    f = (dt - bc0) inv_w and u = f - floor(f) rounded to a multiple of
    2^-b (the kernels accumulate fixed point, fixed_bits); weights outside
    the window are dropped."""
    dt = np.asarray(dt, dtype=np.float64)
    bits = fixed_bits(dt.size)
    f = (dt - bc0) * inv_w
    f = f[(f > -1.0) & (f < n_slices)]
    fl = np.floor(f)
    j = fl.astype(np.int64)
    u = np.ldexp(np.rint(np.ldexp(f - fl, bits)), -bits)
    p = np.zeros(n_slices)
    a = j >= 0
    np.add.at(p, j[a], 1.0 - u[a])
    b = j + 1 < n_slices
    np.add.at(p, j[b] + 1, u[b])
    return p


def resonator_impedance(R, fr, Q, n_fft, bin_size):
    """impedance_sources.py:382-414 / fast_resonator.cpp:19-74 summed and
    divided by the bin size (impedance.py:846-890); Z[0] = 0."""
    R, fr, Q = (np.atleast_1d(np.asarray(x, dtype=np.float64)) for x in (R, fr, Q))
    f = np.arange(1, n_fft // 2 + 1) / (n_fft * bin_size)
    Z = np.zeros(n_fft // 2 + 1, dtype=np.complex128)
    for r in range(len(R)):
        Z[1:] += R[r] / (1 + 1j * Q[r] * (f / fr[r] - fr[r] / f))
    return Z / bin_size


def track(dt0, dE0, V, omega, phi, acc, drift_c, charge, Z, scale, n_slices, n_fft,
          bc0, inv_w):
    """V, omega, phi: (n_turns, n_rf); acc, drift_c: (n_turns,).  Z: the
    impedance (n_fft/2+1) or None; scale = q e ratio.  Returns
    (dt, dE, final profile, induced voltages per turn)."""
    dt = np.array(dt0, dtype=np.float64)
    dE = np.array(dE0, dtype=np.float64)
    p = cic(dt, n_slices, bc0, inv_w)
    vinds = []
    for t in range(len(acc)):
        if Z is not None:
            v = -scale * np.fft.irfft(Z * np.fft.rfft(p, n_fft), n_fft)[:n_slices]
            vinds.append(v)
            f = (dt - bc0) * inv_w
            m = (f >= 0) & (f < n_slices - 1)
            fl = np.floor(f[m])
            k = fl.astype(np.int64)
            u = f[m] - fl
            dE[m] += charge * (v[k] * (1.0 - u) + v[k + 1] * u)
        s = np.zeros_like(dt)
        for j in range(V.shape[1]):
            s += V[t, j] * np.sin(omega[t, j] * dt + phi[t, j])
        dE += charge * s + acc[t]
        dt = dt + drift_c[t] * dE
        p = cic(dt, n_slices, bc0, inv_w)
    return dt, dE, p, vinds


def bunch_loss(profile, target, bin_centers, time_unit=1e-9):
    """RMS bunch length squared (time_unit^2) from the line density with
    trapezoid moments (filters_and_fitting.py:158-172) + L2 mismatch of the
    profile normalised to sum 1 against target."""
    p = np.asarray(profile, dtype=np.float64)
    w = np.ones_like(p)
    w[0] = w[-1] = 0.5
    norm = np.sum(w * p)
    mu = np.sum(w * p * bin_centers) / norm
    sig2 = np.sum(w * p * (bin_centers - mu) ** 2) / norm
    return sig2 / time_unit**2 + np.sum((p / p.sum() - target) ** 2)


def scale_of(charge, intensity, n):
    return charge * E_CHARGE * intensity / n
