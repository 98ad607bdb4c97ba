"""Generate the golden fixtures in tests/golden/ by running the REFERENCE.

Run in a container that holds the reference checkout (BLOND_REFERENCE_ROOT,
by default a checkout named ``reference`` beside this repository) after
``make -C oracle``:

    python tests/golden/gen_golden.py

The reference's Python package is imported with its C++ backend pointed at
oracle/_ref (the reference's own sources compiled with the
``--parallel --optimize`` flag set).  Every fixture stores the inputs it was
made from, so the tests never need the reference at run time.

Fixtures
--------
profile_golden.npz    reference unit-test input dt_coordinates.npz
                      (unittests/beam_profile/test_beam_profile_object.py:
                      52-140) and the three profiles it pins at :169-230.
kernels_{f64,f32}.npz seeded inputs and the reference kernels' outputs
                      (kick, drift x3 solvers, histogram, smooth_histogram,
                      linear_interp_kick, rf_volt_comp, fast_resonator).
machine_c1.npz        Ring/RFStation/bigaussian derived quantities for the
                      26 GeV/c, h=4620, 4.5 MV machine.
track_*.npz           multi-turn runs of the reference objects
                      (RingAndRFTracker, Profile, TotalInducedVoltage).
induced_*.npz         one-turn induced voltages (Freq, Time, Inductive).
nfft_known.npz        n_fft / n_induced_voltage known answers.
wakes_resonator.npz   resonator_induced_voltage_1_turn (butils_wrap_python.py:
                      656-790) on seeded profiles, windows, times and modes.
mtw_resonator.npz     the reference's own multi-turn-wake resonator test
                      (unittests/impedances/test_impedance.py:127-187): its
                      stored expectation mtw_resonator_induced_voltage.npy
                      and the same run repeated here, with the time array.
mtw_tracks.npz        multi-turn wakes in mtw_mode 'time' (InducedVoltageFreq,
                      InducedVoltageTime) tracked over several turns.
profile_fits.npz      Profile fit options 'gaussian', 'rms', 'fwhm'.
beam_phase.npz        the reference's compiled beam_phase / beam_phase_fast.
cut_options.npz       CutOptions.set_cuts without given cuts (default and
                      n_sigma frames) on the unit-test dt and a bigaussian.
beam_feedback.npz     BeamFeedback (every machine type) tracked for 200 turns:
                      per-turn beam phase, phase error, frequency correction,
                      mean dt, the final RF frequency/phase rows and a sample
                      of the final coordinates (the SPS set-up of the
                      reference's unittests/llrf/test_beam_feedback.py:22-59).
"""
from __future__ import annotations

import ctypes as ct
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import ref_harness  # noqa: E402

REF = ref_harness.DEFAULT_REF
blond = ref_harness.import_reference("double")

from blond.beam.beam import Beam, Proton  # noqa: E402
from blond.beam.distributions import bigaussian  # noqa: E402
from blond.beam.profile import (CutOptions, FitOptions, Profile,  # noqa: E402
                                OtherSlicesOptions)
from blond.impedances.impedance import (InducedVoltageFreq,  # noqa: E402
                                        InducedVoltageResonator,
                                        InducedVoltageTime,
                                        InductiveImpedance,
                                        TotalInducedVoltage)
from blond.impedances.impedance_sources import Resonators  # noqa: E402
from blond.input_parameters.rf_parameters import RFStation  # noqa: E402
from blond.input_parameters.ring import Ring  # noqa: E402
from blond.toolbox.next_regular import next_regular  # noqa: E402
from blond.trackers.tracker import RingAndRFTracker  # noqa: E402
from blond.utils import bmath as bm  # noqa: E402


def save(name, **arrays):
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **arrays)
    print(f"wrote {name}: {os.path.getsize(path) / 1024:.1f} KiB")


# --------------------------------------------------------------------------
# 1. reference profile goldens (unittests/beam_profile)
# --------------------------------------------------------------------------
def gen_profile_golden():
    dt = np.load(os.path.join(
        REF, "unittests/beam_profile/dt_coordinates.npz"))["arr_0"]
    ring = Ring(125, 0.001, 1e9, Proton(), 1)
    rf = RFStation(ring=ring, harmonic=[1], voltage=[7e6], phi_rf_d=[0.],
                   n_rf=1)
    beam = Beam(ring, len(dt), 1e10)
    beam.dt = dt
    p1 = Profile(beam)
    p1.track()
    p2 = Profile(beam, cut_options=CutOptions(
        cut_left=0, cut_right=2 * np.pi, n_slices=200, cuts_unit="rad",
        rf_station=rf))
    p3 = Profile(beam, cut_options=CutOptions(
        cut_left=0, cut_right=ring.t_rev[0], n_slices=150, cuts_unit="s"),
        other_slices_options=OtherSlicesOptions(smooth=True,
                                                direct_slicing=False))
    p3.track()
    save("profile_golden.npz", dt=dt,
         cuts1=np.array([p1.cut_left, p1.cut_right]),
         counts1=p1.n_macroparticles,
         cuts2=np.array([p2.cut_left, p2.cut_right]),
         counts2=p2.n_macroparticles,
         cuts3=np.array([p3.cut_left, p3.cut_right]),
         smooth3=p3.n_macroparticles,
         bin_centers1=p1.bin_centers, edges1=p1.edges,
         t_rev=np.array([ring.t_rev[0]]),
         omega_rf0=np.array([rf.omega_rf[0, 0]]))


# --------------------------------------------------------------------------
# 2. raw kernel outputs of the reference's compiled C++
# --------------------------------------------------------------------------
def _kernel_cases(lib, real, tag):
    rng = np.random.default_rng(12345)
    c_real = ct.c_double if real == np.float64 else ct.c_float
    P = lambda a: a.ctypes.data_as(ct.c_void_p)  # noqa: E731
    n = 4099
    out = {}
    t_c = 2.5e-9
    dt = (t_c + 0.4e-9 * rng.standard_normal(n)).astype(real)
    dE = (2.3e7 * rng.standard_normal(n)).astype(real)
    out["dt"] = dt.copy()
    out["dE"] = dE.copy()
    # kick, 2 harmonics
    V = np.array([4.5e6, 0.45e6], real)
    om = np.array([1.2579e9, 4 * 1.2579e9], real)
    ph = np.array([0.0, np.pi], real)
    out["kick_V"], out["kick_omega"], out["kick_phi"] = V, om, ph
    out["kick_charge"] = np.array([1.0])
    out["kick_acc"] = np.array([-1234.5])
    x = dE.copy()
    lib.kick(P(dt), P(x), ct.c_int(2), c_real(1.0), P(V), P(om), P(ph),
             ct.c_int(n), c_real(-1234.5))
    out["kick_dE"] = x
    # drift, all solvers, alpha orders 0..2
    dpar = dict(t_rev=2.3e-5, length_ratio=1.0, eta_0=1.786e-3, eta_1=2.1e-4,
                eta_2=-3.3e-5, alpha_0=1 / 18**2, alpha_1=1.1e-4,
                alpha_2=-2.0e-5, beta=0.99935, energy=26.017e9)
    for k, v in dpar.items():
        out["drift_" + k] = np.array([v])
    for solver in (0, 1, 2):
        for order in (0, 1, 2):
            y = dt.copy()
            lib.drift(P(y), P(dE), ct.c_int(solver),
                      c_real(dpar["t_rev"]), c_real(dpar["length_ratio"]),
                      c_real(order), c_real(dpar["eta_0"]),
                      c_real(dpar["eta_1"]), c_real(dpar["eta_2"]),
                      c_real(dpar["alpha_0"]), c_real(dpar["alpha_1"]),
                      c_real(dpar["alpha_2"]), c_real(dpar["beta"]),
                      c_real(dpar["energy"]), ct.c_int(n))
            out[f"drift_s{solver}_o{order}"] = y
    # histogram / smooth histogram
    for S in (100, 1024, 4096):
        cl, cr = t_c - 1.25e-9, t_c + 1.25e-9
        h = np.zeros(S, real)
        lib.histogram(P(dt), P(h), c_real(cl), c_real(cr), ct.c_int(S),
                      ct.c_int(n))
        out[f"hist_{S}"] = h
        hs = np.zeros(S, real)
        lib.smooth_histogram(P(dt), P(hs), c_real(cl), c_real(cr),
                             ct.c_int(S), ct.c_int(n))
        out[f"smooth_{S}"] = hs
    out["hist_cuts"] = np.array([t_c - 1.25e-9, t_c + 1.25e-9])
    # linear interp kick
    S = 257
    edges = np.linspace(t_c - 1.25e-9, t_c + 1.25e-9, S + 1).astype(real)
    bc = ((edges[:-1] + edges[1:]) / 2).astype(real)
    volt = (1e5 * np.sin(np.linspace(0, 7, S)) + 3e4).astype(real)
    out["lik_bc"], out["lik_V"] = bc, volt
    z = dE.copy()
    lib.linear_interp_kick(P(dt), P(z), P(volt), P(bc), c_real(1.0),
                           ct.c_int(S), ct.c_int(n), c_real(-77.0))
    out["lik_dE"] = z
    out["lik_acc"] = np.array([-77.0])
    # rf_volt_comp
    rv = np.zeros(S, real)
    lib.rf_volt_comp(P(V), P(om), P(ph), P(bc), ct.c_int(2), ct.c_int(S),
                     P(rv))
    out["rfv"] = rv
    # fast resonator
    nf = 513
    freq = np.fft.rfftfreq(1024, 2.5e-9 / 1024).astype(real)
    R = np.array([5e6, 1e5, 3e4], real)
    Q = np.array([1.0, 200.0, 3e4], real)
    fr = np.array([1e9, 200e6, 1.4e9], real)
    re = np.zeros(nf, real)
    im = np.zeros(nf, real)
    lib.fast_resonator_real_imag(P(re), P(im), P(freq), P(R), P(Q), P(fr),
                                 ct.c_int(3), ct.c_int(nf))
    out.update(res_freq=freq, res_R=R, res_Q=Q, res_fr=fr, res_re=re,
               res_im=im)
    save(f"kernels_{tag}.npz", **out)


def gen_kernels():
    for tag, real in (("f64", np.float64), ("f32", np.float32)):
        lib = ct.CDLL(os.path.join(ROOT, "oracle", "_ref",
                                   f"libblond_ref_{'double' if tag == 'f64' else 'single'}.so"))
        _kernel_cases(lib, real, tag)


# --------------------------------------------------------------------------
# 3. machine quantities and bunch generation
# --------------------------------------------------------------------------
def c1_machine(n_turns=1000, harmonics=(4620,), voltages=(4.5e6,),
               phases=(0.0,)):
    ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), n_turns)
    rf = RFStation(ring, list(harmonics), list(voltages), list(phases),
                   n_rf=len(harmonics))
    return ring, rf


def gen_machine():
    ring, rf = c1_machine()
    beam = Beam(ring, 10000, 1e10)
    bigaussian(ring, rf, beam, 0.4e-9, seed=0)
    ring2, rf2 = c1_machine(100, (4620, 4 * 4620), (4.5e6, 0.45e6),
                            (0.0, np.pi))
    save("machine_c1.npz",
         t_rev=ring.t_rev[:3], beta=ring.beta[0, :3], gamma=ring.gamma[0, :3],
         energy=ring.energy[0, :3], momentum=ring.momentum[0, :3],
         eta_0=ring.eta_0[0, :3], eta_1=ring.eta_1[0, :3],
         eta_2=ring.eta_2[0, :3], delta_E=ring.delta_E[0, :3],
         omega_rf=rf.omega_rf[:, :3], phi_rf=rf.phi_rf[:, :3],
         phi_s=rf.phi_s[:3], t_rf=rf.t_rf[:, :3], Q_s=rf.Q_s[:3],
         sigma_dE=np.array([beam.sigma_dE]), dt=beam.dt, dE=beam.dE,
         omega_rf_2=rf2.omega_rf[:, :3], phi_s_2=rf2.phi_s[:3])


# --------------------------------------------------------------------------
# 4. multi-turn tracking with the reference objects
# --------------------------------------------------------------------------
def _window(rf, half=1.25e-9):
    t_c = (rf.phi_s[0] - rf.phi_rf[0, 0]) / rf.omega_rf[0, 0]
    return t_c - half, t_c + half


def _track(name, n, n_slices, n_turns, *, harmonics=(4620,),
           voltages=(4.5e6,), phases=(0.0,), solver="simple",
           impedance=None, intensity=1e10, interpolation=False,
           smooth=False, seed=0, sigma_dt=0.4e-9, save_every=1,
           alpha_1=None):
    if alpha_1 is None:
        ring, rf = c1_machine(n_turns, harmonics, voltages, phases)
    else:
        ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), n_turns,
                    alpha_1=alpha_1)
        rf = RFStation(ring, list(harmonics), list(voltages), list(phases),
                       n_rf=len(harmonics))
    beam = Beam(ring, n, intensity)
    # bigaussian matches sigma_dE with the first harmonic only
    bigaussian(ring, rf, beam, sigma_dt, seed=seed)
    dt0, dE0 = beam.dt.copy(), beam.dE.copy()
    cl, cr = _window(rf)
    profile = Profile(beam, CutOptions(cut_left=cl, cut_right=cr,
                                       n_slices=n_slices),
                      other_slices_options=OtherSlicesOptions(smooth=smooth))
    tiv = None
    if impedance is not None:
        kind, args = impedance
        if kind == "freq":
            src = Resonators(*args)
            ivs = [InducedVoltageFreq(beam, profile, [src])]
        elif kind == "freq+ind":
            src = Resonators(*args[0])
            ivs = [InducedVoltageFreq(beam, profile, [src]),
                   InductiveImpedance(beam, profile,
                                      [args[1]] * (n_turns + 1), rf)]
        elif kind == "time":
            src = Resonators(*args)
            ivs = [InducedVoltageTime(beam, profile, [src])]
        tiv = TotalInducedVoltage(beam, profile, ivs)
        tiv.induced_voltage_sum()
    tracker = RingAndRFTracker(rf, beam, solver=solver,
                               interpolation=interpolation,
                               profile=profile if interpolation else None,
                               total_induced_voltage=tiv
                               if interpolation else None)
    profiles, vinds = [profile.n_macroparticles.copy()], []
    for turn in range(n_turns):
        if tiv is not None and not interpolation:
            tiv.track()
            vinds.append(tiv.induced_voltage.copy())
        elif tiv is not None:
            tiv.induced_voltage_sum()
            vinds.append(tiv.induced_voltage.copy())
        tracker.track()
        profile.track()
        if (turn + 1) % save_every == 0:
            profiles.append(profile.n_macroparticles.copy())
    arrays = dict(dt0=dt0, dE0=dE0, dt=beam.dt, dE=beam.dE,
                  profiles=np.array(profiles),
                  cuts=np.array([cl, cr]), bin_centers=profile.bin_centers,
                  n_turns=np.array([n_turns]), n_slices=np.array([n_slices]),
                  intensity=np.array([intensity]),
                  harmonics=np.array(harmonics, float),
                  voltages=np.array(voltages), phases=np.array(phases),
                  solver=np.array([solver]), save_every=np.array([save_every]))
    if vinds:
        arrays["vind"] = np.array(vinds)
    if impedance is not None:
        arrays["n_fft"] = np.array([ivs[0].n_fft])
        arrays["total_impedance"] = ivs[0].total_impedance
    save(name, **arrays)


def gen_tracks():
    _track("track_rf.npz", 5000, 100, 50)
    _track("track_exact.npz", 3000, 100, 10, solver="exact")
    _track("track_legacy.npz", 3000, 100, 10, solver="legacy")
    _track("track_legacy_a1.npz", 3000, 100, 10, solver="legacy",
           alpha_1=1e-4)
    _track("track_full.npz", 5000, 1024, 20,
           impedance=("freq", (5e6, 1e9, 1.0)))
    _track("track_double_rf.npz", 4000, 512, 20,
           harmonics=(4620, 4 * 4620), voltages=(4.5e6, 0.45e6),
           phases=(0.0, np.pi),
           impedance=("freq", ([1e5, 3e4, 1e4], [200e6, 800e6, 1.4e9],
                               [100.0, 3000.0, 30000.0])))
    _track("track_interp.npz", 4000, 256, 10, interpolation=True,
           impedance=("freq", (5e6, 1e9, 1.0)))
    _track("track_time.npz", 3000, 200, 5,
           impedance=("time", (5e6, 1e9, 1.0)))
    _track("track_inductive.npz", 3000, 256, 5,
           impedance=("freq+ind", ((5e6, 1e9, 1.0), 0.1)))
    _track("track_smooth.npz", 3000, 128, 5, smooth=True,
           impedance=("freq", (5e6, 1e9, 1.0)))


# --------------------------------------------------------------------------
# 5. n_fft known answers (unittests/impedances/test_impedance.py:30-125)
# --------------------------------------------------------------------------
def gen_nfft():
    prof = Profile(None, cut_options=CutOptions(cut_left=0, cut_right=5e-9,
                                                n_slices=16))
    src = Resonators([4.5e6], [200.222e6], [200])
    a = InducedVoltageFreq(None, prof, [src])
    b = InducedVoltageFreq(None, prof, [src], frequency_resolution=3e6)
    c = InducedVoltageTime(None, prof, [src])
    d = InducedVoltageTime(None, prof, [src], wake_length=11e-9)
    targets = np.arange(1, 5000)
    save("nfft_known.npz",
         freq_default=np.array([a.n_fft, a.n_induced_voltage]),
         freq_res3e6=np.array([b.n_fft, b.n_induced_voltage]),
         time_default=np.array([c.n_fft, c.n_induced_voltage]),
         time_wake11ns=np.array([d.n_fft, d.n_induced_voltage]),
         freq_res3e6_impedance=b.total_impedance,
         time_wake11ns_impedance=d.total_impedance,
         next_regular_targets=targets,
         next_regular_values=np.array([next_regular(int(t))
                                       for t in targets]))


# --------------------------------------------------------------------------
# 6. time-domain wakes: resonator convolution, multi-turn wakes, fits
# --------------------------------------------------------------------------
def gen_wakes_resonator():
    from blond.utils.butils_wrap_python import resonator_induced_voltage_1_turn
    rng = np.random.default_rng(2024)
    out = {}
    cases = [
        # name, n_slices, bin_size, modes (R, f_r, Q), times
        ("narrow", 512, 1.5e-12, ([1.19e10], [1.2973e9], [0.696e6]), "mtw3"),
        ("two", 256, 2.5e-11, ([5e6, 1e6], [1e9, 3e9], [1.0, 30.0]), "window"),
        ("lowq", 300, 1e-11, ([1e6], [5e9], [0.6]), "outside"),
        ("many", 128, 5e-11, ([1e5, 3e4, 1e4, 2e3], [200e6, 800e6, 1.4e9, 2.1e9],
                              [100.0, 3000.0, 30000.0, 2.0]), "window"),
    ]
    for name, S, bs, (R, fr, Q), kind in cases:
        edges = np.linspace(0.0, S * bs, S + 1)
        bc = (edges[1:] + edges[:-1]) / 2
        n_mp = 200000
        x = rng.normal(0.5 * S * bs, 0.12 * S * bs, n_mp)
        prof = np.histogram(x, S, (0.0, S * bs))[0].astype(np.float64)
        if kind == "mtw3":
            t = np.concatenate([2e-5 * k + np.linspace(bc[0], bc[-1], S)
                                for k in range(3)])
        elif kind == "outside":
            t = np.concatenate([bc, bc[0] - 20 * bs + np.arange(3 * S) * 0.37 * bs])
        else:
            t = bc.copy()
        R = np.array(R, float)
        om = 2 * np.pi * np.array(fr, float)
        Q = np.array(Q, float)
        Qt = Q * np.sqrt(1.0 - 1.0 / (4.0 * Q ** 2.0))
        nt = len(t)
        v, _ = resonator_induced_voltage_1_turn(
            np.zeros(S - 1), prof, bc, bs, nt, np.zeros((nt, S)), t,
            om * Qt / Q, om / (2.0 * Q), Qt, len(R), om, Q,
            np.ones((len(R), nt)), 1.0, n_mp, 1e11 / n_mp, R, np.zeros(nt),
            np.float64)
        for k, a in dict(profile=prof, bin_centers=bc, bin_size=np.array([bs]),
                         n_macroparticles=np.array([n_mp]), time=t, R=R,
                         omega_r=om, Q=Q, ratio=np.array([1e11 / n_mp]),
                         voltage=v).items():
            out[f"{name}_{k}"] = a
    out["names"] = np.array([c[0] for c in cases])
    save("wakes_resonator.npz", **out)


def gen_mtw_resonator():
    import importlib.util
    path = os.path.join(REF, "unittests/impedances/test_impedance.py")
    spec = importlib.util.spec_from_file_location("ref_impedance_test", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    case = mod.TestInducedVoltageResonatorMultiTurnWake()
    case.setUp()
    ivr = InducedVoltageResonator(beam=case.beam, profile=case.profile,
                                  multi_turn_wake=True, resonators=case.resonator,
                                  rf_station=case.rf_station,
                                  time_decay_factor=0.00001)
    tiv = TotalInducedVoltage(beam=case.beam, profile=case.profile,
                              induced_voltage_list=[ivr])
    tracker = RingAndRFTracker(rf_station=case.rf_station, beam=case.beam,
                               profile=case.profile, total_induced_voltage=tiv,
                               interpolation=True)
    time_array = ivr.time_array.copy()
    volts, full, dts, dEs = [], [], [], []
    for _ in range(case.n_turns):
        tiv.induced_voltage_sum()
        full.append(ivr.induced_voltage.copy())
        tracker.track()
        volts.append(tiv.induced_voltage.copy())
        dts.append(case.beam.dt.copy())
        dEs.append(case.beam.dE.copy())
    expected = np.load(os.path.join(
        REF, "unittests/impedances/data/mtw_resonator_induced_voltage.npy"))
    np.testing.assert_allclose(np.array(volts), expected, rtol=1e-5, atol=1e-1)
    save("mtw_resonator.npz", expected=expected, rerun=np.array(volts),
         full=np.array(full), time_array=time_array,
         n_mtw_memory=np.array([ivr.n_mtw_memory]),
         profile=case.profile.n_macroparticles.copy(),
         bin_centers=case.profile.bin_centers.copy(),
         fit=np.asarray(case.profile.fit_extra_options, float),
         t_rev=case.ring.t_rev.copy(), phi_s=case.rf_station.phi_s.copy(),
         omega_rf=case.rf_station.omega_rf[:, :2].copy(),
         dt=np.array(dts), dE=np.array(dEs))


def _small_ring_mtw(kind, n_turns=6, n=5000, S=64, seed=3):
    """A 30 m ring (t_rev ~ 100 ns) whose wake memory spans three turns."""
    ring = Ring(30.0, 0.02, 2e9, Proton(), n_turns)
    rf = RFStation(ring, [4], [20e3], [0.0], n_rf=1)
    beam = Beam(ring, n, 5e11)
    bigaussian(ring, rf, beam, 2e-9, seed=seed)
    dt0, dE0 = beam.dt.copy(), beam.dE.copy()
    t_rf = rf.t_rf[0, 0]
    profile = Profile(beam, CutOptions(cut_left=0.0, cut_right=t_rf, n_slices=S))
    src = Resonators([2e4], [4.2 * 4 / ring.t_rev[0]], [60.0])
    wake = 3 * ring.t_rev[0]
    if kind == "freq":
        iv = InducedVoltageFreq(beam, profile, [src],
                                frequency_resolution=1 / wake,
                                multi_turn_wake=True, rf_station=rf,
                                mtw_mode="time")
    else:
        iv = InducedVoltageTime(beam, profile, [src], wake_length=wake,
                                multi_turn_wake=True, rf_station=rf,
                                mtw_mode="time")
    tiv = TotalInducedVoltage(beam, profile, [iv])
    tracker = RingAndRFTracker(rf, beam)
    vinds, mems, profiles = [], [], [profile.n_macroparticles.copy()]
    for _ in range(n_turns):
        tiv.track()
        vinds.append(tiv.induced_voltage.copy())
        mems.append(iv.mtw_memory.copy())
        tracker.track()
        profile.track()
        profiles.append(profile.n_macroparticles.copy())
    return dict(dt0=dt0, dE0=dE0, dt=beam.dt.copy(), dE=beam.dE.copy(),
                vind=np.array(vinds), memory=np.array(mems),
                profiles=np.array(profiles), n_fft=np.array([iv.n_fft]),
                n_induced_voltage=np.array([iv.n_induced_voltage]),
                time_mtw=iv.time_mtw, t_rev=ring.t_rev.copy(),
                cuts=np.array([profile.cut_left, profile.cut_right]))


def gen_mtw_tracks():
    out = {}
    for kind in ("freq", "time"):
        for k, a in _small_ring_mtw(kind).items():
            out[f"{kind}_{k}"] = a
    save("mtw_tracks.npz", **out)


def gen_profile_fits():
    ring, rf = c1_machine(10)
    beam = Beam(ring, 20000, 1e10)
    bigaussian(ring, rf, beam, 0.4e-9, seed=7)
    cl, cr = _window(rf)
    out = dict(dt=beam.dt.copy(), cuts=np.array([cl, cr]), n_slices=np.array([200]))
    out["bin_centers"] = Profile(beam, CutOptions(cut_left=cl, cut_right=cr,
                                                  n_slices=200)).bin_centers.copy()
    for opt in ("gaussian", "rms", "fwhm"):
        p = Profile(beam, CutOptions(cut_left=cl, cut_right=cr, n_slices=200),
                    FitOptions(fit_option=opt))
        out[f"{opt}_position"] = np.array([p.bunchPosition])
        out[f"{opt}_length"] = np.array([p.bunchLength])
        if opt == "gaussian":
            out["gaussian_params"] = np.asarray(p.fit_extra_options, float)
            out["p0"] = np.array([p.n_macroparticles.max(), beam.dt.mean(),
                                  beam.dt.std()])
        out["profile"] = p.n_macroparticles.copy()
    save("profile_fits.npz", **out)


# --------------------------------------------------------------------------
# 7. beam-phase loop
# --------------------------------------------------------------------------
BF_CASES = {
    # name: (machine set-up, configuration, delay)
    "LHC": ("sps", {"machine": "LHC", "PL_gain": 1000.0}, 0),
    "LHC_window": ("sps", {"machine": "LHC", "PL_gain": 1000.0,
                           "window_coefficient": 2e8, "time_offset": 2.55e-9}, 0),
    "LHC_SL": ("lhc", {"machine": "LHC", "PL_gain": 500.0, "SL_gain": 50.0}, 0),
    "LHC_F": ("sps", {"machine": "LHC_F", "PL_gain": 1000.0, "FL_gain": 0.05}, 5),
    "SPS_F": ("sps", {"machine": "SPS_F", "PL_gain": 1000.0, "FL_gain": 0.05}, 0),
    "SPS_F_window": ("sps", {"machine": "SPS_F", "PL_gain": 1000.0, "FL_gain": 0.05,
                             "window_coefficient": -1 / 5.1e-9,
                             "time_offset": 2.5e-9}, 0),
    "SPS_RL": ("sps", {"machine": "SPS_RL", "PL_gain": 1000.0, "RL_gain": 1e6,
                       "sample_dE": 3}, 0),
    "PSB": ("sps", {"machine": "PSB", "PL_gain": 1000.0, "RL_gain": [1e4, 1e2],
                    "period": 1e-4}, 0),
    # with a broadband resonator (1e11 protons): induced voltage + loop per turn
    "LHC_F_Z": ("sps", {"machine": "LHC_F", "PL_gain": 1000.0, "FL_gain": 0.05}, 0),
    "SPS_RL_Z": ("sps", {"machine": "SPS_RL", "PL_gain": 1000.0, "RL_gain": 1e6,
                         "sample_dE": 2}, 0),
}
BF_IMPEDANCE = {"LHC_F_Z", "SPS_RL_Z"}
BF_TURNS = 200
BF_PARTICLES = 200000


def bf_machine(kind, n_turns=BF_TURNS):
    """The SPS set-up of test_beam_feedback.py:22-59 (bunch 0.05 ns, moved
    by 0.1 ns) or an LHC-like ring (450 GeV/c, h=35640, 6 MV) whose
    synchrotron frequency suits the LHC synchro loop."""
    if kind == "sps":
        ring = Ring(6911.5038, 1.0 / 17.95142852 ** 2, 25.92e9, Proton(), n_turns)
        rf = RFStation(ring, 4620, 4.5e6, 0)
        sigma, shift = 0.05e-9, 0.1e-9
    else:
        ring = Ring(26658.883, 3.225e-4, 450e9, Proton(), n_turns)
        rf = RFStation(ring, 35640, 6e6, 0)
        sigma, shift = 0.25e-9, 0.2e-9
    return ring, rf, sigma, shift


def gen_beam_phase():
    """The reference's compiled beam_phase / beam_phase_fast
    (cpp_routines/beam_phase.cpp:6-65) on seeded profiles, both precisions."""
    out = {}
    for tag, real, c_real in (("f64", np.float64, ct.c_double), ("f32", np.float32, ct.c_float)):
        lib = ct.CDLL(os.path.join(ROOT, "oracle", "_ref",
                                   f"libblond_ref_{'double' if tag == 'f64' else 'single'}.so"))
        lib.beam_phase.restype = c_real
        lib.beam_phase_fast.restype = c_real
        rng = np.random.default_rng(777)
        P = lambda a: a.ctypes.data_as(ct.c_void_p)  # noqa: E731
        vals = []
        for k, n in enumerate((1024, 333, 4096, 2)):
            bc = np.linspace(0.0, 5e-9, n + 1)[:-1].astype(real) + real(2.5e-9 / n)
            prof = np.maximum(0, 1e4 * np.exp(-((bc - 2.6e-9) / 0.3e-9) ** 2)
                              + rng.normal(0, 20, n)).astype(real)
            prm = (2e8 * (k - 1), 1.2583e9 + 10 * k, 0.01 * k, 5e-9 / n)
            a = lib.beam_phase(P(bc), P(prof), c_real(prm[0]), c_real(prm[1]),
                               c_real(prm[2]), c_real(prm[3]), ct.c_int(n))
            f = lib.beam_phase_fast(P(bc), P(prof), c_real(prm[1]), c_real(prm[2]),
                                    c_real(prm[3]), ct.c_int(n))
            out[f"{tag}_{k}_bc"], out[f"{tag}_{k}_profile"] = bc, prof
            out[f"{tag}_{k}_params"] = np.array(prm)
            vals.append((a, f))
        out[f"{tag}_coeff"] = np.array(vals)
    save("beam_phase.npz", **out)


def gen_beam_feedback():
    from blond.llrf.beam_feedback import BeamFeedback
    from blond.trackers.tracker import FullRingAndRF
    # BeamFeedback.beam_phase_sharpWindow (SPS_F) calls bm.trapz and
    # bm.logical_and, which no backend of the reference defines
    # (utils/bmath_backends.py); numpy's functions of those names are
    # provided here.
    for name, fn in (("trapz", np.trapezoid), ("logical_and", np.logical_and)):
        if not hasattr(bm, name):
            setattr(bm, name, fn)
    out = {"names": np.array(list(BF_CASES))}
    for name, (kind, cfg, delay) in BF_CASES.items():
        ring, rf, sigma, shift = bf_machine(kind)
        z = name in BF_IMPEDANCE
        beam = Beam(ring, BF_PARTICLES, 1e11 if z else 1.2e6)
        bigaussian(ring, rf, beam, sigma, seed=1234)
        beam.dt += shift
        profile = Profile(beam, CutOptions(cut_left=0, cut_right=rf.t_rf[0, 0],
                                           n_slices=1024))
        cfg = {k: (list(v) if isinstance(v, list) else v) for k, v in cfg.items()}
        loop = BeamFeedback(ring, rf, profile, cfg, delay=delay)
        section = RingAndRFTracker(rf, beam, profile=profile, beam_feedback=loop)
        tracker = FullRingAndRF([section])
        tiv = None
        if z:
            tiv = TotalInducedVoltage(beam, profile, [InducedVoltageFreq(
                beam, profile, [Resonators(5e6, 1e9, 1.0)])])
        trace = np.zeros((BF_TURNS, 4))
        for turn in range(BF_TURNS):
            trace[turn, 0] = np.mean(beam.dt)
            if z:
                # the fused engine's order: induced kick, RF turn, slicing
                tiv.track()
                tracker.track()
                profile.track()
            else:
                profile.track()
                tracker.track()
            trace[turn, 1:] = (loop.phi_beam, loop.dphi, loop.domega_rf)
        out[f"{name}_trace"] = trace
        out[f"{name}_omega_rf"] = rf.omega_rf[0].copy()
        out[f"{name}_phi_rf"] = rf.phi_rf[0].copy()
        out[f"{name}_dt"] = beam.dt[::997].copy()
        out[f"{name}_dE"] = beam.dE[::997].copy()
    save("beam_feedback.npz", **out)


def gen_cut_options():
    """CutOptions.set_cuts (beam/profile.py:175-211) without given cuts --
    the default frame (min/max -/+ 5 %) and n_sigma frames -- on the
    reference's unit-test dt and on a seeded bigaussian bunch."""
    dt_unit = np.load(os.path.join(
        REF, "unittests/beam_profile/dt_coordinates.npz"))["arr_0"]
    ring, rf = c1_machine(10)
    bunch = Beam(ring, 20000, 1e10)
    bigaussian(ring, rf, bunch, 0.4e-9, seed=11)
    # the unit-test dt is profile_golden.npz's `dt`
    out = {"dt_bunch": np.array(bunch.dt)}
    for name, dt in (("unit", dt_unit), ("bunch", np.array(bunch.dt))):
        b = Beam(ring, len(dt), 1e10)
        b.dt = dt
        for tag, kw in (("default", {}), ("nsigma3", {"n_sigma": 3}),
                        ("nsigma55", {"n_sigma": 5.5})):
            co = CutOptions(n_slices=64, **kw)
            co.set_cuts(b)
            out[f"{name}_{tag}"] = np.array([co.cut_left, co.cut_right])
            out[f"{name}_{tag}_bc"] = np.array(co.bin_centers)
    save("cut_options.npz", **out)


def run_reference_profile_test():
    """Run the reference's own profile unit test (its literal expected
    counts) against oracle/_ref before the fixture is trusted."""
    import importlib.util
    import unittest
    path = os.path.join(REF, "unittests/beam_profile/test_beam_profile_object.py")
    spec = importlib.util.spec_from_file_location("ref_profile_test", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    suite = unittest.TestLoader().loadTestsFromTestCase(mod.testProfileClass)
    res = unittest.TextTestRunner(verbosity=0).run(suite)
    assert res.wasSuccessful(), "reference profile test failed on oracle/_ref"


if __name__ == "__main__":
    bm.use_cpp()
    if len(sys.argv) > 1:  # only the named generators, e.g. gen_cut_options
        for name in sys.argv[1:]:
            globals()[name]()
        sys.exit(0)
    run_reference_profile_test()
    gen_profile_golden()
    gen_kernels()
    gen_machine()
    gen_tracks()
    gen_nfft()
    gen_wakes_resonator()
    gen_mtw_resonator()
    gen_mtw_tracks()
    gen_profile_fits()
    gen_beam_phase()
    gen_beam_feedback()
