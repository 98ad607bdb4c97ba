"""CPU checks of the differentiable map's restatement (oracle/adjoint_oracle.py).

With the induced voltage off, its kick and drift are the reference's
formulas: it must agree with the reference-pinned oracle (cpu_oracle,
itself checked against the reference's fixtures).  Its cloud-in-cell
profile is checked against a particle-by-particle loop, and its gradient
definitions against the closed form of a one-turn case.
"""
import numpy as np

import adjoint_oracle as ao
import cpu_oracle as co
from conftest import normwise
from blond_b200.beam.beam import Proton
from blond_b200.beam.distributions import _get_dE_from_dt, bigaussian_arrays
from blond_b200.input_parameters.rf_parameters import RFStation
from blond_b200.input_parameters.ring import Ring


def machine(T):
    ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), T)
    rf = RFStation(ring, [4620], [4.5e6], [0.0])
    return ring, rf


def programmes(rf, T):
    V = np.asarray(rf.voltage, float)[:, :T].T.copy()
    om = np.asarray(rf.omega_rf, float)[:, :T].T.copy()
    ph = np.asarray(rf.phi_rf, float)[:, :T].T.copy()
    acc = -np.asarray(rf.delta_E, float)[:T]
    nx = slice(1, T + 1)
    c = (np.asarray(rf.t_rev, float)[nx] * rf.length_ratio * np.asarray(rf.eta_0, float)[nx]
         / (np.asarray(rf.beta, float)[nx] ** 2 * np.asarray(rf.energy, float)[nx]))
    return V, om, ph, acc, c


def test_kick_drift_match_reference_pinned_oracle():
    T, n, S = 25, 20000, 100
    ring, rf = machine(T)
    centre = (rf.phi_s[0] - rf.phi_rf[0, 0]) / rf.omega_rf[0, 0]
    dt0, dE0 = bigaussian_arrays(n, 0.4e-9, _get_dE_from_dt(ring, rf, 0.4e-9), centre, 1)
    cl, cr = centre - 1.25e-9, centre + 1.25e-9
    w = (cr - cl) / S
    V, om, ph, acc, c = programmes(rf, T)
    dt, dE, _, _ = ao.track(dt0, dE0, V, om, ph, acc, c, 1.0, None, 0.0, S, S, cl + w / 2,
                            1 / w)
    edges = np.linspace(cl, cr, S + 1)
    odt, odE, _, _ = co.track_oracle(dt0, dE0, ring, rf, (cl, cr), (edges[:-1] + edges[1:]) / 2,
                                     S, T)
    assert normwise(dt, odt) < 1e-12 and normwise(dE, odE) < 1e-12


def test_cic_against_loop():
    rng = np.random.default_rng(0)
    S, bc0, inv_w = 16, 1.0, 2.0
    dt = rng.uniform(0.0, 10.0, 3000)
    dt[:3] = [bc0, bc0 + (S - 1) / inv_w, np.nan]
    p = ao.cic(dt, S, bc0, inv_w)
    q = np.zeros(S)
    for x in dt:
        f = (x - bc0) * inv_w
        if not (-1 < f < S):
            continue
        j = int(np.floor(f))
        bits = ao.fixed_bits(len(dt))
        u = round((f - j) * 2**bits) / 2**bits  # fixed-point weights
        if j >= 0:
            q[j] += 1 - u
        if j + 1 < S:
            q[j + 1] += u
    np.testing.assert_allclose(p, q, rtol=0, atol=1e-12)
    # every particle between the first and last bin centre keeps weight 1
    f = (dt - bc0) * inv_w
    assert abs(p.sum() - np.sum((f >= 0) & (f <= S - 1))
               - sum(1 - abs(x) if -1 < x < 0 else S - x if S - 1 < x < S else 0
                     for x in f if x == x and not (0 <= x <= S - 1) and -1 < x < S)) < 1e-9


def test_cic_is_continuous():
    """The property the adjoint relies on: moving a particle across a bin
    centre or edge changes the profile by O(step)."""
    S, bc0, inv_w = 32, 0.0, 1.0
    for x in (3.0, 3.5, 7.25, 0.0, 30.999):
        a = ao.cic(np.array([x - 1e-9]), S, bc0, inv_w)
        b = ao.cic(np.array([x + 1e-9]), S, bc0, inv_w)
        assert np.abs(a - b).max() < 1e-8


def test_resonator_impedance_matches_fast_resonator():
    n_fft, bs = 256, 2.5e-9 / 256
    f = np.fft.rfftfreq(n_fft, bs)
    R, fr, Q = np.array([5e6, 1e5]), np.array([1e9, 2e8]), np.array([1.0, 300.0])
    Z = co.fast_resonator(R, Q, f, fr) / bs
    assert normwise(ao.resonator_impedance(R, fr, Q, n_fft, bs), Z) < 1e-14
