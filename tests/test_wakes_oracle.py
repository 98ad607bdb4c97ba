"""CPU checks of the time-domain wake restatement (oracle/wakes_oracle.py)
and of the host logic around the wake kernels.

* The oracle's resonator convolution against the reference's own outputs
  (tests/golden/wakes_resonator.npz) and its multi-turn memory against the
  reference's multi-turn-wake resonator test (mtw_resonator.npz).
* The bin recurrence that blond_b200/csrc/wakes.cu evaluates, restated in
  numpy here, against the oracle's time x bin sum: the identity the kernel
  rests on, checked without a GPU.
* The multi-turn time array and the FWHM fit helper of the drop-in
  classes, bit for bit against the reference's.
"""
import numpy as np
import pytest

import wakes_oracle as wo
from conftest import golden, normwise
from blond_b200.beam.profile import _fwhm, _gauss
from blond_b200.impedances.impedance import mtw_resonator_time_array


def _cases():
    g = golden("wakes_resonator.npz")
    for name in g["names"]:
        yield str(name), {k[len(name) + 1:]: g[k] for k in g.files
                          if k.startswith(f"{name}_")}


@pytest.mark.parametrize("name", [n for n, _ in _cases()])
def test_oracle_resonator_matches_reference(name):
    c = dict(_cases())[name]
    v = wo.resonator_induced_voltage(c["profile"], c["bin_centers"], c["bin_size"][0],
                                     int(c["n_macroparticles"][0]), c["time"], c["R"],
                                     c["omega_r"], c["Q"], 1.0, c["ratio"][0])
    assert normwise(v, c["voltage"]) < 1e-14


def recurrence(profile, bc, bin_size, N, t, R, omega_r, Q, charge, ratio):
    """The kernel's algorithm: J_i = e^{p h_i} J_{i-1} - kappa_{i-1}
    expm1(p h_i); V_j = scale sum_r coef_r (Re[c e^{p (t_j - bc_i)}
    (J_i - kappa_i)] + 2 kappa_i), i = #{bc < t_j} - 1."""
    S = len(bc)
    kap = np.zeros(S)
    kap[:-1] = np.diff(profile) / np.diff(bc) / (N * bin_size)
    qt, a, b = wo.resonator_constants(omega_r, Q)
    m = np.searchsorted(bc, t, side="left")
    out = np.zeros(len(t))
    for r in range(len(R)):
        p = complex(-b[r], a[r])
        J = np.zeros(S, complex)
        for i in range(1, S):
            h = bc[i] - bc[i - 1]
            J[i] = np.exp(p * h) * J[i - 1] - kap[i - 1] * np.expm1(p * h)
        ok = m > 0
        i = m[ok] - 1
        O = np.exp(p * (t[ok] - bc[i])) * (J[i] - kap[i])
        val = np.zeros(len(t))
        val[ok] = 2 * O.real + O.imag / qt[r] + 2 * kap[i]
        out += R[r] / (2 * omega_r[r] * Q[r]) * val
    return out * (-charge * wo.E_CHARGE * N * ratio)


@pytest.mark.parametrize("name", [n for n, _ in _cases()])
def test_recurrence_matches_direct_sum(name):
    c = dict(_cases())[name]
    args = (c["profile"], c["bin_centers"], c["bin_size"][0], int(c["n_macroparticles"][0]),
            c["time"], c["R"], c["omega_r"], c["Q"], 1.0, c["ratio"][0])
    v = recurrence(*args)
    ref = c["voltage"]
    bc = c["bin_centers"]
    inside = c["time"] <= bc[-1] + (bc[1] - bc[0])
    # inside the window the two sums agree to rounding; later turns carry
    # the reference's own rounding of a * (t - bc) at |a t| ~ 1e5 rad
    assert normwise(v[inside], ref[inside]) < 1e-12
    assert normwise(v, ref) < 1e-8


def test_mtw_time_array_bit_exact():
    g = golden("mtw_resonator.npz")
    bc = g["bin_centers"]
    # impedance.py:1159-1169 with the test's Q / omega_R and decay factor
    Q, omega = 0.696e6, 2 * np.pi * (1297263703 - 1320)
    decay_turns = np.ceil(np.log(1e-5) / np.log(wo.E_CHARGE) * 2 * Q / omega
                          / np.min(g["t_rev"]))
    n_turns = min(int(decay_turns), 3)
    min_index = int(np.abs(bc[0] - g["phi_s"][0] / g["omega_rf"][0, 0]).argmin())
    t = mtw_resonator_time_array(bc, len(bc), g["t_rev"], n_turns, min_index)
    np.testing.assert_array_equal(t, g["time_array"])


def test_oracle_mtw_replays_reference_test():
    """The reference's test tracks a beam at rest whose profile is sliced
    once: every turn convolves the same profile, and the memory adds up."""
    g = golden("mtw_resonator.npz")
    bc, t = g["bin_centers"], g["time_array"]
    S = len(bc)
    bin_size = bc[1] - bc[0]
    v1 = wo.resonator_induced_voltage(g["profile"], bc, bin_size, 1001, t,
                                      [11897424000.0], [2 * np.pi * (1297263703 - 1320)],
                                      [0.696e6], 1.0, 1e10 / 1001)
    mem = np.zeros(int(g["n_mtw_memory"][0]))
    for turn in range(3):
        mem, iv = wo.resonator_mtw(mem, v1, S)
        assert normwise(iv, g["full"][turn]) < 1e-12
        np.testing.assert_allclose(iv[:S], g["expected"][turn], rtol=1e-5, atol=1e-1)


def test_fwhm_and_gauss_helpers_match_reference():
    g = golden("profile_fits.npz")
    bp, bl = _fwhm(g["profile"], g["bin_centers"])
    assert bp == g["fwhm_position"][0]
    assert bl == g["fwhm_length"][0]
    x = np.linspace(-3, 3, 7)
    np.testing.assert_array_equal(_gauss(x, 2.0, 0.5, 1.5),
                                  2.0 * np.exp(-((x - 0.5) ** 2) / 2.0 / 1.5 ** 2))
