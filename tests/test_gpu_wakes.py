"""Time-domain wakes on the device vs the reference.

* blond_interp_f64 against numpy.interp, bit for bit.
* blond_resonator_induced_voltage_f64 against the reference's
  resonator_induced_voltage_1_turn outputs (tests/golden/wakes_resonator.npz)
  and the oracle's time x bin sum.  Bars: 1e-12 of max|V| inside the
  slicing window; 1e-8 over later turns, where the reference's own
  rounding of a * (t - bc) at |a t| ~ 1e5 rad is the larger error.
* InducedVoltageResonator with multi_turn_wake=True replaying the
  reference's unit test (unittests/impedances/test_impedance.py:127-187)
  against its stored expectation, at the test's own tolerance and at 1e-8
  against the same run repeated with the reference.
* InducedVoltageFreq / InducedVoltageTime multi-turn wakes (mtw_mode
  'time') tracked over six turns against the reference objects.
* Profile fit options against the reference's fits.
"""
import ctypes as ct

import numpy as np
import pytest
import torch

import wakes_oracle as wo
from conftest import golden, normwise
from blond_b200 import _lib
from blond_b200 import bmath as bm
from blond_b200.beam.beam import Beam, Proton
from blond_b200.beam.profile import CutOptions, FitOptions, Profile
from blond_b200.engine import FusedTracker
from blond_b200.impedances.impedance import (InducedVoltageFreq,
                                             InducedVoltageResonator,
                                             InducedVoltageTime,
                                             TotalInducedVoltage)
from blond_b200.impedances.impedance_sources import Resonators
from blond_b200.input_parameters.rf_parameters import RFStation
from blond_b200.input_parameters.ring import Ring
from blond_b200.trackers.tracker import RingAndRFTracker

pytestmark = pytest.mark.gpu

E = wo.E_CHARGE


def dev(a):
    return torch.as_tensor(np.asarray(a, dtype=np.float64), device="cuda")


# ---------------------------------------------------------------- interp
def test_interp_bit_exact_vs_numpy(cuda):
    rng = np.random.default_rng(5)
    xp = np.sort(rng.uniform(-1, 1, 1000))
    fp = rng.normal(size=1000)
    x = np.concatenate([rng.uniform(-1.2, 1.2, 20000), xp[::7], [xp[0], xp[-1]],
                        [-5.0, 5.0, np.nan]])
    for left, right in ((None, None), (0.0, 0.0), (-7.5, 3.25)):
        got = bm.interp(dev(x), dev(xp), dev(fp), left=left, right=right).cpu().numpy()
        want = np.interp(x, xp, fp, left=left, right=right)
        np.testing.assert_array_equal(got, want)


def test_interp_shift_uniform_grid_and_single_point(cuda):
    # the multi-turn-wake shift: memory(t + t_rev) on its own time grid
    tm = np.linspace(0, 3e-7, 768, endpoint=False)
    mem = np.random.default_rng(1).normal(size=768)
    for trev in (1.1053409e-07, 0.0, 2.9e-7, 4e-7):
        got = bm.interp(dev(tm), dev(tm), dev(mem), left=0, right=0, x_shift=trev)
        np.testing.assert_array_equal(got.cpu().numpy(),
                                      np.interp(tm + trev, tm, mem, left=0, right=0))
    x = np.array([-1.0, 0.5, 1.0, 2.0])
    got = bm.interp(dev(x), dev([0.5]), dev([3.0])).cpu().numpy()
    np.testing.assert_array_equal(got, np.interp(x, [0.5], [3.0]))


def test_interp_rejects_aliased_output(cuda):
    xp, fp = dev(np.arange(8.0)), dev(np.arange(8.0))
    P = lambda t: ct.c_void_p(t.data_ptr())  # noqa: E731
    with pytest.raises(_lib.BlondB200Error):
        _lib.call("blond_interp_f64", P(xp), 8, 0.0, P(xp), P(fp), 8, 0.0, 0.0, 0,
                  P(fp), None)
    torch.cuda.synchronize()


# ---------------------------------------------------- resonator convolution
def _cases():
    g = golden("wakes_resonator.npz")
    for name in g["names"]:
        yield str(name), {k[len(name) + 1:]: g[k] for k in g.files
                          if k.startswith(f"{name}_")}


@pytest.mark.parametrize("name", [n for n, _ in _cases()])
def test_resonator_kernel_matches_reference(cuda, name):
    c = dict(_cases())[name]
    N = int(c["n_macroparticles"][0])
    scale = -1.0 * E * N * c["ratio"][0]
    v, _ = bm.resonator_induced_voltage(dev(c["profile"]), dev(c["bin_centers"]),
                                        c["bin_size"][0], N, dev(c["time"]), c["R"],
                                        c["omega_r"], c["Q"], scale)
    v = v.cpu().numpy()
    bc = c["bin_centers"]
    inside = c["time"] <= bc[-1] + (bc[1] - bc[0])
    assert normwise(v[inside], c["voltage"][inside]) < 1e-12
    assert normwise(v, c["voltage"]) < 1e-8


def test_resonator_kernel_uneven_bins_and_rows(cuda):
    """Increasing but uneven bin centres, several modes, per-mode rows."""
    rng = np.random.default_rng(11)
    S = 700
    bc = np.cumsum(rng.uniform(0.5e-11, 1.5e-11, S))
    prof = np.maximum(0, 1000 * np.exp(-((bc - bc.mean()) / (0.15 * bc[-1])) ** 2)
                      + rng.normal(0, 5, S))
    t = np.concatenate([bc, np.linspace(bc[0] - 1e-10, bc[-1] + 3e-9, 2000)])
    R, om, Q = [3e5, 1e4, 2e6], 2 * np.pi * np.array([4e8, 1.9e9, 6e9]), [5.0, 400.0, 0.55]
    want, rows = wo.resonator_induced_voltage(prof, bc, 1e-11, 123456, t, R, om, Q,
                                              1.0, 10.0, per_resonator=True)
    tmp = torch.zeros((3, len(t)), dtype=torch.float64, device="cuda")
    v, _ = bm.resonator_induced_voltage(dev(prof), dev(bc), 1e-11, 123456, dev(t), R, om, Q,
                                        -1.0 * E * 123456 * 10.0, tmp_matrix=tmp)
    assert normwise(v.cpu().numpy(), want) < 1e-12
    for r in range(3):
        assert normwise(tmp[r].cpu().numpy(), rows[r]) < 1e-12


def test_resonator_reference_signature(cuda):
    c = dict(_cases())["two"]
    S, nt = len(c["bin_centers"]), len(c["time"])
    kappa = torch.zeros(S - 1, dtype=torch.float64, device="cuda")
    deltaT = torch.zeros((nt, S), dtype=torch.float64, device="cuda")
    tmp = torch.ones((2, nt), dtype=torch.float64, device="cuda")
    iv = torch.zeros(nt, dtype=torch.float64, device="cuda")
    N = int(c["n_macroparticles"][0])
    Qt, a, b = wo.resonator_constants(c["omega_r"], c["Q"])
    v, dT = bm.resonator_induced_voltage_1_turn(
        kappa, dev(c["profile"]), dev(c["bin_centers"]), c["bin_size"][0], nt, deltaT,
        dev(c["time"]), a, b, Qt, 2, c["omega_r"], c["Q"], tmp, 1.0, N, c["ratio"][0],
        c["R"], iv, np.float64)
    assert v is iv and dT is deltaT
    assert normwise(v.cpu().numpy(), c["voltage"]) < 1e-12
    np.testing.assert_array_equal(
        kappa.cpu().numpy(),
        np.diff(c["profile"]) / np.diff(c["bin_centers"]) / (N * c["bin_size"][0]))
    np.testing.assert_array_equal(deltaT.cpu().numpy(),
                                  c["time"][:, None] - c["bin_centers"][None, :])
    rows = tmp.cpu().numpy()
    assert normwise(rows.sum(axis=0) * (-E * N * c["ratio"][0]), c["voltage"]) < 1e-12


def test_resonator_mtw_fused_matches_separate_steps(cuda):
    """memory_out = memory_in moved by one window + V, bit for bit the
    reference's append / slice / add on the same V."""
    c = dict(_cases())["narrow"]
    N, S = int(c["n_macroparticles"][0]), len(c["bin_centers"])
    scale = -1.0 * E * N * c["ratio"][0]
    args = (dev(c["profile"]), dev(c["bin_centers"]), c["bin_size"][0], N, dev(c["time"]),
            c["R"], c["omega_r"], c["Q"], scale)
    v, _ = bm.resonator_induced_voltage(*args)
    n_t = len(c["time"])
    for n_mem in (n_t, n_t + 1, n_t + 3 * S):
        mem = dev(np.random.default_rng(n_mem).normal(size=n_mem) * 1e5)
        new, _ = bm.resonator_induced_voltage(*args, memory_in=mem, shift=S)
        want = torch.cat((mem, mem.new_zeros(S)))[S:].clone()
        want[:n_t] += v
        assert torch.equal(new, want)
    with pytest.raises(_lib.BlondB200Error):
        bm.resonator_induced_voltage(*args, memory_in=dev(np.zeros(n_t - 1)), shift=S)
    torch.cuda.synchronize()


def test_resonator_argument_checks(cuda):
    bc, p, t = dev(np.arange(1.0, 9.0)), dev(np.ones(8)), dev(np.arange(4.0))
    with pytest.raises(_lib.BlondB200Error):
        bm.resonator_induced_voltage(p, bc, 1.0, 8, t, [1.0], [1.0], [0.4], 1.0)
    with pytest.raises(_lib.BlondB200Error):
        bm.resonator_induced_voltage(p, bc, 1.0, 8, t, [1.0] * 65, [1.0] * 65, [1.0] * 65,
                                     1.0)
    small = torch.empty(16, dtype=torch.uint8, device="cuda")
    with pytest.raises(_lib.BlondB200Error):
        bm.resonator_induced_voltage(p, bc, 1.0, 8, t, [1.0], [1.0], [1.0], 1.0,
                                     workspace=small)
    with pytest.raises(ValueError):
        bm.resonator_induced_voltage_1_turn(None, p, dev(np.arange(8.0)[::-1].copy()), 1.0,
                                            4, None, t, None, None, None, 1, [1.0], [1.0],
                                            None, 1.0, 8, 1.0, [1.0], None, np.float64)
    torch.cuda.synchronize()


# ------------------------------------------------- InducedVoltageResonator
def mtw_test_machine():
    """unittests/impedances/test_impedance.py:129-165."""
    ring = Ring(ring_length=np.full(1, 5989.95), alpha_0=np.full(1, 4.68e-4),
                particle=Proton(), n_turns=3, n_sections=1,
                synchronous_data=np.array([25e9, 25e9, 1.04 * 25e9, 1.05 * 25e9]))
    h = int(1297263703 * ring.t_rev[0])
    rf = RFStation(ring=ring, harmonic=[h], voltage=[3e9], phi_rf_d=[0.0], n_rf=1)
    beam = Beam(ring, 1001, int(1e10))
    prof = Profile(beam, CutOptions(cut_left=0, cut_right=2 * np.pi, n_slices=2 ** 9,
                                    cuts_unit="rad", rf_station=rf),
                   FitOptions(fit_option="gaussian"))
    res = Resonators(11897424000, 1297263703 - 1320, 0.696e6)
    return ring, rf, beam, prof, res


def test_mtw_resonator_reference_unit_test(cuda):
    g = golden("mtw_resonator.npz")
    ring, rf, beam, prof, res = mtw_test_machine()
    np.testing.assert_allclose(prof.fit_extra_options, g["fit"], rtol=1e-6)
    ivr = InducedVoltageResonator(beam=beam, profile=prof, multi_turn_wake=True,
                                  resonators=res, rf_station=rf,
                                  time_decay_factor=0.00001)
    np.testing.assert_array_equal(np.asarray(ivr.time_array), g["time_array"])
    assert ivr.n_mtw_memory == int(g["n_mtw_memory"][0])
    tiv = TotalInducedVoltage(beam=beam, profile=prof, induced_voltage_list=[ivr])
    tracker = RingAndRFTracker(rf_station=rf, beam=beam, profile=prof,
                               total_induced_voltage=tiv, interpolation=True)
    volts = []
    for turn in range(3):
        tiv.induced_voltage_sum()
        assert normwise(ivr.induced_voltage.cpu().numpy(), g["full"][turn]) < 1e-8
        tracker.track()
        volts.append(tracker.totalInducedVoltage.induced_voltage.cpu().numpy())
        assert normwise(beam.dt.cpu().numpy(), g["dt"][turn]) < 1e-12
        assert normwise(beam.dE.cpu().numpy(), g["dE"][turn]) < 1e-8
    volts = np.array(volts)
    # the reference test's own assertion (test_impedance.py:186)
    np.testing.assert_allclose(volts, g["expected"], rtol=1e-5, atol=1e-1)
    assert normwise(volts, g["rerun"]) < 1e-8


def test_resonator_one_turn_matches_oracle(cuda):
    g = golden("track_interp.npz")
    ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), 5)
    rf = RFStation(ring, [4620], [4.5e6], [0.0])
    beam = Beam(ring, len(g["dt0"]), 1e10, dt=g["dt0"], dE=g["dE0"])
    cl, cr = g["cuts"]
    prof = Profile(beam, CutOptions(cut_left=cl, cut_right=cr, n_slices=256))
    res = Resonators([5e6, 2e5], [1e9, 2.3e9], [1.0, 50.0])
    t_user = np.linspace(cl - 1e-9, cr + 4e-9, 3001)
    for time_array in (None, t_user):
        ivr = InducedVoltageResonator(beam, prof, res, time_array=time_array)
        ivr.induced_voltage_1turn()
        t = prof.bin_centers if time_array is None else time_array
        want = wo.resonator_induced_voltage(prof.n_macroparticles.cpu().numpy(),
                                            prof.bin_centers, prof.bin_size,
                                            beam.n_macroparticles, t, res.R_S, res.omega_R,
                                            res.Q, 1.0, beam.ratio)
        assert normwise(ivr.induced_voltage.cpu().numpy(), want) < 1e-12
    tiv = TotalInducedVoltage(beam, prof, [InducedVoltageResonator(beam, prof, res)])
    tiv.track()  # the kick through linear_interp_kick runs on the device too
    with pytest.raises(NotImplementedError):
        FusedTracker(RingAndRFTracker(rf, beam), prof, tiv, precision="f64")


# --------------------------------------------- FFT wakes with 'time' memory
def small_ring(g, kind, n_turns=6):
    ring = Ring(30.0, 0.02, 2e9, Proton(), n_turns)
    rf = RFStation(ring, [4], [20e3], [0.0], n_rf=1)
    beam = Beam(ring, len(g[f"{kind}_dt0"]), 5e11, dt=g[f"{kind}_dt0"], dE=g[f"{kind}_dE0"])
    cl, cr = g[f"{kind}_cuts"]
    prof = Profile(beam, CutOptions(cut_left=cl, cut_right=cr, n_slices=64))
    src = Resonators([2e4], [4.2 * 4 / ring.t_rev[0]], [60.0])
    wake = 3 * ring.t_rev[0]
    if kind == "freq":
        iv = InducedVoltageFreq(beam, prof, [src], frequency_resolution=1 / wake,
                                multi_turn_wake=True, rf_station=rf, mtw_mode="time")
    else:
        iv = InducedVoltageTime(beam, prof, [src], wake_length=wake,
                                multi_turn_wake=True, rf_station=rf, mtw_mode="time")
    return ring, rf, beam, prof, iv


@pytest.mark.parametrize("kind", ["freq", "time"])
def test_mtw_time_mode_tracks_reference(cuda, kind):
    g = golden("mtw_tracks.npz")
    ring, rf, beam, prof, iv = small_ring(g, kind)
    assert iv.n_fft == int(g[f"{kind}_n_fft"][0])
    np.testing.assert_array_equal(iv.time_mtw.cpu().numpy(), g[f"{kind}_time_mtw"])
    tiv = TotalInducedVoltage(beam, prof, [iv])
    tracker = RingAndRFTracker(rf, beam)
    profiles = [prof.n_macroparticles.cpu().numpy()]
    for turn in range(6):
        tiv.track()
        assert normwise(tiv.induced_voltage.cpu().numpy(), g[f"{kind}_vind"][turn]) < 1e-10
        assert normwise(iv.mtw_memory.cpu().numpy(), g[f"{kind}_memory"][turn]) < 1e-10
        tracker.track()
        prof.track()
        profiles.append(prof.n_macroparticles.cpu().numpy())
    assert normwise(beam.dt.cpu().numpy(), g[f"{kind}_dt"]) < 1e-11
    assert normwise(beam.dE.cpu().numpy(), g[f"{kind}_dE"]) < 1e-11
    np.testing.assert_array_equal(np.array(profiles), g[f"{kind}_profiles"])
    with pytest.raises(NotImplementedError):
        FusedTracker(tracker, prof, tiv, precision="f64")


def test_mtw_freq_mode_needs_buffer_extra(cuda):
    """The reference's 'freq' memory reads an attribute nothing sets
    (impedance.py:419); without it the constructor fails the same way."""
    g = golden("mtw_tracks.npz")
    ring = Ring(30.0, 0.02, 2e9, Proton(), 6)
    rf = RFStation(ring, [4], [20e3], [0.0], n_rf=1)
    beam = Beam(ring, len(g["freq_dt0"]), 5e11, dt=g["freq_dt0"], dE=g["freq_dE0"])
    prof = Profile(beam, CutOptions(cut_left=0.0, cut_right=rf.t_rf[0, 0], n_slices=64))
    with pytest.raises(AttributeError):
        InducedVoltageFreq(beam, prof, [Resonators([2e4], [1.5e8], [60.0])],
                           frequency_resolution=1 / (3 * ring.t_rev[0]),
                           multi_turn_wake=True, rf_station=rf, mtw_mode="freq")


# ---------------------------------------------------------------- fits
@pytest.mark.parametrize("option", ["gaussian", "rms", "fwhm"])
def test_profile_fits_match_reference(cuda, option):
    g = golden("profile_fits.npz")
    ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), 10)
    dt = g["dt"]
    beam = Beam(ring, len(dt), 1e10, dt=dt, dE=np.zeros_like(dt))
    cl, cr = g["cuts"]
    prof = Profile(beam, CutOptions(cut_left=cl, cut_right=cr, n_slices=200),
                   FitOptions(fit_option=option))
    np.testing.assert_array_equal(prof.n_macroparticles.cpu().numpy(), g["profile"])
    rtol = {"gaussian": 1e-6, "rms": 1e-12, "fwhm": 0}[option]
    np.testing.assert_allclose(prof.bunchPosition, g[f"{option}_position"][0], rtol=rtol)
    np.testing.assert_allclose(prof.bunchLength, g[f"{option}_length"][0], rtol=rtol)
