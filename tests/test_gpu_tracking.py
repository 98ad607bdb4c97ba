"""Multi-turn tracking through the drop-in objects and the fused engine vs
the reference's own objects (fixtures from tests/golden/gen_golden.py).

Bars (FP64): dt/dE within 1e-11 normwise after the fixture's turns (1e-12
per turn, the single-turn bar, does not compound visibly over <= 50
turns; legacy/exact solvers 1e-10 because the fixture came from the
reference's fast-math build, see test_oracle_golden), profiles bit-exact,
induced voltage within 1e-10 normwise.
"""
import numpy as np
import pytest
import torch

from conftest import golden, normwise
from blond_b200.beam.beam import Beam, Proton
from blond_b200.beam.profile import CutOptions, OtherSlicesOptions, Profile
from blond_b200.engine import FusedTracker
from blond_b200.impedances.impedance import (InducedVoltageFreq,
                                             InducedVoltageTime,
                                             InductiveImpedance,
                                             TotalInducedVoltage)
from blond_b200.impedances.impedance_sources import Resonators
from blond_b200.input_parameters.rf_parameters import RFStation
from blond_b200.input_parameters.ring import Ring
from blond_b200.trackers.tracker import RingAndRFTracker

pytestmark = pytest.mark.gpu

SOLVERS = {"simple": 0, "legacy": 1, "exact": 2}


def build(g, alpha_1=None):
    nt = int(g["n_turns"][0])
    ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), nt, alpha_1=alpha_1)
    h = [float(x) for x in g["harmonics"]]
    rf = RFStation(ring, h, list(g["voltages"]), list(g["phases"]), n_rf=len(h))
    beam = Beam(ring, len(g["dt0"]), float(g["intensity"][0]), dt=g["dt0"], dE=g["dE0"])
    return ring, rf, beam


def make_profile(g, beam, smooth=False):
    cl, cr = g["cuts"]
    return Profile(beam, CutOptions(cut_left=cl, cut_right=cr,
                                    n_slices=int(g["n_slices"][0])),
                   other_slices_options=OtherSlicesOptions(smooth=smooth))


def impedance_objects(name, beam, prof, rf):
    if name in ("track_full.npz", "track_interp.npz", "track_smooth.npz"):
        return [InducedVoltageFreq(beam, prof, [Resonators(5e6, 1e9, 1.0)])]
    if name == "track_double_rf.npz":
        return [InducedVoltageFreq(beam, prof, [Resonators(
            [1e5, 3e4, 1e4], [200e6, 800e6, 1.4e9], [100.0, 3000.0, 30000.0])])]
    if name == "track_time.npz":
        return [InducedVoltageTime(beam, prof, [Resonators(5e6, 1e9, 1.0)])]
    if name == "track_inductive.npz":
        return [InducedVoltageFreq(beam, prof, [Resonators(5e6, 1e9, 1.0)]),
                InductiveImpedance(beam, prof, [0.1] * (rf.n_turns + 1), rf)]
    return None


CASES = ["track_rf.npz", "track_exact.npz", "track_legacy.npz",
         "track_legacy_a1.npz", "track_full.npz", "track_double_rf.npz",
         "track_interp.npz", "track_time.npz", "track_inductive.npz",
         "track_smooth.npz"]


@pytest.mark.parametrize("name", CASES)
def test_dropin_objects_match_reference(cuda, name):
    g = golden(name)
    ring, rf, beam = build(g, alpha_1=1e-4 if name == "track_legacy_a1.npz" else None)
    smooth = name == "track_smooth.npz"
    prof = make_profile(g, beam, smooth)
    ivs = impedance_objects(name, beam, prof, rf)
    tiv = TotalInducedVoltage(beam, prof, ivs) if ivs else None
    interp = name == "track_interp.npz"
    if tiv is not None:
        tiv.induced_voltage_sum()
        assert normwise(ivs[0].total_impedance.cpu().numpy(), g["total_impedance"]) < 1e-13
    tracker = RingAndRFTracker(rf, beam, solver=str(g["solver"][0]),
                               interpolation=interp, profile=prof if interp else None,
                               total_induced_voltage=tiv if interp else None)
    vinds, profiles = [], [prof.n_macroparticles.cpu().numpy()]
    for _ in range(int(g["n_turns"][0])):
        if tiv is not None:
            if interp:
                tiv.induced_voltage_sum()
            else:
                tiv.track()
            vinds.append(tiv.induced_voltage.cpu().numpy())
        tracker.track()
        prof.track()
        profiles.append(prof.n_macroparticles.cpu().numpy())
    tol = 1e-10 if str(g["solver"][0]) != "simple" else 1e-11
    assert normwise(beam.dt.cpu().numpy(), g["dt"]) < tol
    assert normwise(beam.dE.cpu().numpy(), g["dE"]) < tol
    if smooth:
        assert normwise(np.array(profiles), g["profiles"]) < 1e-10
    else:
        np.testing.assert_array_equal(np.array(profiles), g["profiles"])
    if vinds:
        assert normwise(np.array(vinds), g["vind"]) < 1e-10
    assert rf.counter[0] == int(g["n_turns"][0])


FUSED = ["track_rf.npz", "track_exact.npz", "track_legacy.npz", "track_full.npz",
         "track_double_rf.npz", "track_time.npz", "track_inductive.npz"]


@pytest.mark.parametrize("name", FUSED)
@pytest.mark.parametrize("turns_per_graph", [1, 3])
@pytest.mark.parametrize("kernel", ["tma", "plain"])
def test_fused_engine_matches_reference(cuda, name, turns_per_graph, kernel):
    g = golden(name)
    ring, rf, beam = build(g)
    prof = make_profile(g, beam)
    ivs = impedance_objects(name, beam, prof, rf)
    tiv = TotalInducedVoltage(beam, prof, ivs) if ivs else None
    tracker = RingAndRFTracker(rf, beam, solver=str(g["solver"][0]))
    fused = FusedTracker(tracker, prof, tiv, precision="f64",
                         turns_per_graph=turns_per_graph, kernel=kernel)
    nt = int(g["n_turns"][0])
    np.testing.assert_array_equal(fused.profile_tensor().cpu().numpy(), g["profiles"][0])
    fused.track(nt - 1)
    if tiv is not None:
        # induced voltage of the last tracked turn's head
        assert normwise(fused.induced_voltage_tensor().cpu().numpy(), g["vind"][nt - 2]) < 1e-10
    np.testing.assert_array_equal(fused.profile_tensor().cpu().numpy(), g["profiles"][nt - 1])
    fused.track(1)
    tol = 1e-10 if str(g["solver"][0]) != "simple" else 1e-11
    assert normwise(beam.dt.cpu().numpy(), g["dt"]) < tol
    assert normwise(beam.dE.cpu().numpy(), g["dE"]) < tol
    np.testing.assert_array_equal(fused.profile_tensor().cpu().numpy(), g["profiles"][-1])
    fused.sync()
    np.testing.assert_array_equal(prof.n_macroparticles.cpu().numpy(), g["profiles"][-1])
    assert rf.counter[0] == nt


def test_fused_engine_rejects_turns_beyond_programme(cuda):
    from blond_b200 import BlondB200Error
    g = golden("track_rf.npz")
    ring, rf, beam = build(g)
    prof = make_profile(g, beam)
    fused = FusedTracker(RingAndRFTracker(rf, beam), prof)
    with pytest.raises(BlondB200Error):
        fused.track(int(g["n_turns"][0]) + 1)


def test_fused_odd_particle_count_and_ragged_tail(cuda):
    """n odd exercises the scalar tail of the pair loop."""
    g = golden("track_full.npz")
    n = 4999
    ring, rf, _ = build(g)
    beam = Beam(ring, n, float(g["intensity"][0]), dt=g["dt0"][:n], dE=g["dE0"][:n])
    prof = make_profile(g, beam)
    tiv = TotalInducedVoltage(beam, prof, [InducedVoltageFreq(beam, prof, [Resonators(5e6, 1e9, 1.0)])])
    import cpu_oracle as o
    odt, odE, oprof, _ = o.track_oracle(
        g["dt0"][:n], g["dE0"][:n], ring, rf, tuple(g["cuts"]), g["bin_centers"],
        int(g["n_slices"][0]), 5,
        impedance=(tiv.induced_voltage_list[0].n_fft,
                   tiv.induced_voltage_list[0].total_impedance.cpu().numpy()),
        intensity=float(g["intensity"][0]) * n / n)
    fused = FusedTracker(RingAndRFTracker(rf, beam), prof, tiv)
    fused.track(5)
    assert normwise(beam.dt.cpu().numpy(), odt) < 1e-12
    assert normwise(beam.dE.cpu().numpy(), odE) < 1e-12
    np.testing.assert_array_equal(fused.profile_tensor().cpu().numpy(), oprof[-1])


@pytest.mark.parametrize("n", [1, 1000, 2048, 2048 * 149 + 7, 2048 * 300 + 1])
@pytest.mark.parametrize("kernel", ["tma", "plain"])
def test_fused_chunk_boundaries(cuda, n, kernel):
    """Particle counts below one 2048-particle chunk, exactly one chunk, more
    chunks than SMs, and ragged tails, against the oracle (3 turns)."""
    import cpu_oracle as o
    from blond_b200.beam.distributions import _get_dE_from_dt, bigaussian_arrays
    ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), 3)
    rf = RFStation(ring, [4620], [4.5e6], [0.0])
    centre = (rf.phi_s[0] - rf.phi_rf[0, 0]) / rf.omega_rf[0, 0]
    dt0, dE0 = bigaussian_arrays(n, 0.4e-9, _get_dE_from_dt(ring, rf, 0.4e-9), centre, 7)
    intensity = 2e6 * n  # the charge per macro-particle of the golden runs
    beam = Beam(ring, n, intensity, dt=dt0, dE=dE0)
    prof = Profile(beam, CutOptions(cut_left=centre - 1.25e-9, cut_right=centre + 1.25e-9,
                                    n_slices=512))
    iv = InducedVoltageFreq(beam, prof, [Resonators(5e6, 1e9, 1.0)])
    tiv = TotalInducedVoltage(beam, prof, [iv])
    fused = FusedTracker(RingAndRFTracker(rf, beam), prof, tiv, kernel=kernel,
                         turns_per_graph=2)
    fused.track(3)
    fused.check()
    odt, odE, oprof, _ = o.track_oracle(
        dt0, dE0, ring, rf, (prof.cut_left, prof.cut_right), prof.bin_centers, 512, 3,
        impedance=(iv.n_fft, iv.total_impedance.cpu().numpy()), intensity=intensity)
    # normwise against the bunch's scale: a handful of particles can all sit
    # near dE = 0, where a per-particle relative error means nothing
    dt_scale = max(np.max(np.abs(odt)), 1e-9)
    dE_scale = max(np.max(np.abs(odE)), 2e7)
    assert np.max(np.abs(beam.dt.cpu().numpy() - odt)) / dt_scale < 1e-12
    assert np.max(np.abs(beam.dE.cpu().numpy() - odE)) / dE_scale < 1e-12
    np.testing.assert_array_equal(fused.profile_tensor().cpu().numpy(), oprof[-1])


def test_fused_mixed_precision_bunch_statistics(cuda):
    """F32P64 (dE float32, RF phase and drift in float64) vs the FP64
    oracle after 200 turns: relative error of the rms bunch length and
    energy spread within 1e-5 (the chosen form's bar)."""
    import cpu_oracle as o
    from blond_b200.beam.distributions import _get_dE_from_dt, bigaussian_arrays
    n, turns = 200000, 200
    ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), turns)
    rf = RFStation(ring, [4620], [4.5e6], [0.0])
    centre = (rf.phi_s[0] - rf.phi_rf[0, 0]) / rf.omega_rf[0, 0]
    dt0, dE0 = bigaussian_arrays(n, 0.4e-9, _get_dE_from_dt(ring, rf, 0.4e-9), centre, 0)
    beam = Beam(ring, n, 1e10, dt=dt0, dE=dE0)
    prof = Profile(beam, CutOptions(cut_left=centre - 1.25e-9, cut_right=centre + 1.25e-9,
                                    n_slices=1024))
    iv = InducedVoltageFreq(beam, prof, [Resonators(5e6, 1e9, 1.0)])
    tiv = TotalInducedVoltage(beam, prof, [iv])
    fused = FusedTracker(RingAndRFTracker(rf, beam), prof, tiv, precision="f32p64")
    fused.track(turns)
    fused.sync()
    odt, odE, _, _ = o.track_oracle(
        dt0, dE0, ring, rf, (prof.cut_left, prof.cut_right), prof.bin_centers, 1024, turns,
        impedance=(iv.n_fft, iv.total_impedance.cpu().numpy()), intensity=1e10)
    dt, dE = beam.dt.cpu().numpy(), beam.dE.cpu().numpy()
    inwin = lambda x: x[(odt > prof.cut_left) & (odt < prof.cut_right)]  # noqa: E731
    for a, b in ((dt, odt), (dE, odE)):
        assert abs(np.std(inwin(a)) / np.std(inwin(b)) - 1) < 1e-5



def test_fused_sharded_api_with_one_rank_matches_unsharded(cuda):
    """The sharded step-by-step path (caller-owned histogram, NCCL
    all-reduce after every particle pass) on a one-rank process group gives
    the graph-replayed path's result bit for bit."""
    import datetime
    import socket
    import torch.distributed as dist
    g = golden("track_full.npz")
    results = []
    for sharded in (False, True):
        ring, rf, beam = build(g)
        prof = make_profile(g, beam)
        tiv = TotalInducedVoltage(beam, prof, impedance_objects("track_full.npz", beam, prof, rf))
        group = None
        if sharded:
            with socket.socket() as s:
                s.bind(("127.0.0.1", 0))
                port = s.getsockname()[1]
            dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0,
                                    world_size=1, timeout=datetime.timedelta(seconds=60))
            group = dist.group.WORLD
        try:
            fused = FusedTracker(RingAndRFTracker(rf, beam), prof, tiv, process_group=group,
                                 turns_per_graph=4)
            fused.track(int(g["n_turns"][0]))
            fused.check()
            results.append((beam.dt.cpu().numpy(), beam.dE.cpu().numpy(),
                            fused.profile_tensor().cpu().numpy()))
        finally:
            if sharded:
                dist.destroy_process_group()
    for a, b in zip(*results):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(results[1][2], g["profiles"][-1])


def _long_profile_case(precision, inductive, turns, n=300001, S=65536):
    """Double RF, four resonators (+ inductive Z/n = 0.1 Ohm) on 2^16
    slices: a profile too long for a shared-memory histogram, so the
    particle kernel deposits into the global one."""
    import cpu_oracle as o
    from blond_b200.beam.distributions import _get_dE_from_dt, bigaussian_arrays
    ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), turns)
    rf = RFStation(ring, [4620, 4 * 4620], [4.5e6, 0.45e6], [0.0, np.pi], n_rf=2)
    centre = (rf.phi_s[0] - rf.phi_rf[0, 0]) / rf.omega_rf[0, 0]
    with pytest.warns(UserWarning):
        sdE = _get_dE_from_dt(ring, rf, 0.4e-9)
    dt0, dE0 = bigaussian_arrays(n, 0.4e-9, sdE, centre, 5)
    beam = Beam(ring, n, 1e11, dt=dt0, dE=dE0)
    prof = Profile(beam, CutOptions(cut_left=centre - 1.25e-9, cut_right=centre + 1.25e-9,
                                    n_slices=S))
    iv = InducedVoltageFreq(beam, prof, [Resonators([2e5, 1e5, 5e4, 3e4],
                                                    [200e6, 800e6, 1.4e9, 2.0e9],
                                                    [100.0, 1000.0, 3000.0, 30000.0])])
    objs = [iv]
    if inductive:
        objs.append(InductiveImpedance(beam, prof, [0.1] * (turns + 1), rf))
    tiv = TotalInducedVoltage(beam, prof, objs)
    fused = FusedTracker(RingAndRFTracker(rf, beam), prof, tiv, precision=precision)
    fused.track(turns)
    fused.sync()
    ref = o.track_oracle(
        dt0, dE0, ring, rf, (prof.cut_left, prof.cut_right), prof.bin_centers, S, turns,
        impedance=(iv.n_fft, iv.total_impedance.cpu().numpy()), intensity=1e11,
        inductive=[0.1] * (turns + 1) if inductive else None)
    return fused, beam, ref


@pytest.mark.parametrize("precision", ["f64", "f32p64"])
def test_fused_2e16_slices_global_histogram(cuda, precision):
    """Three turns on 2^16 slices (FFT length 65536) against the oracle:
    FP64 to 1e-12 with exact counts; F32P64 counts may move by a few
    particles."""
    fused, beam, (odt, odE, oprof, ovind) = _long_profile_case(precision, False, 3)
    dt, dE = beam.dt.cpu().numpy(), beam.dE.cpu().numpy()
    got = fused.profile_tensor().cpu().numpy()
    if precision == "f64":
        assert normwise(dt, odt) < 1e-12 and normwise(dE, odE) < 1e-12
        np.testing.assert_array_equal(got, oprof[-1])
        assert normwise(fused.induced_voltage_tensor().cpu().numpy(), ovind[-1]) < 1e-10
    else:
        # bins are 38 fs wide: the float32 energy moves ~1e-3 of the
        # particles into a neighbouring bin
        assert normwise(dt, odt) < 1e-7
        inwin = (odt > fused.profile.cut_left) & (odt < fused.profile.cut_right)
        for a, b in ((dt, odt), (dE, odE)):
            assert abs(np.std(a[inwin]) / np.std(b[inwin]) - 1) < 1e-5
        assert got.sum() == oprof[-1].sum()
        assert np.abs(got - oprof[-1]).sum() <= 0.01 * len(dt)


def test_fused_2e16_slices_inductive(cuda):
    """One FP64 turn of the same machine with the inductive term added.
    With ~5 macro-particles per bin the derivative of the profile makes
    |V_ind| ~1e8 V and interpolation slopes ~5e21 V/s; the reference's
    kick form dE += dt*slope + (qV - bc*slope) (linear_interp_kick.cpp)
    then cancels terms of max|bc*slope| ~1e13 eV, so one ulp of the induced
    voltage moves dE by ~1e-3 eV.  The bar is therefore a few ulps of that
    term, |dE - dE_oracle| <= 4e-15 max|bc*slope|."""
    fused, beam, (odt, odE, oprof, ovind) = _long_profile_case("f64", True, 1)
    vind = fused.induced_voltage_tensor().cpu().numpy()
    assert normwise(vind, ovind[-1]) < 1e-12
    np.testing.assert_array_equal(fused.profile_tensor().cpu().numpy(), oprof[-1])
    bc = np.asarray(fused.profile.bin_centers)
    slope = np.diff(ovind[-1]) * (len(bc) - 1) / (bc[-1] - bc[0])
    bound = 4e-15 * np.abs(bc[:-1] * slope).max()
    assert np.abs(beam.dE.cpu().numpy() - odE).max() <= bound
    assert normwise(beam.dt.cpu().numpy(), odt) < 1e-10


@pytest.mark.parametrize("precision", ["f64", "f32p64"])
def test_packed_histogram_counter_wraps(cuda, precision):
    """2^16 slices take the packed 16-bit block histogram.  5e7 frozen
    particles (no RF voltage, dE = 0: the coordinates never move), 45% in
    bin 100 and 45% in bin 100 + 2^15 -- the two counters of one shared
    word -- so every block wraps both counters more than once, and the
    low counter's carries run into the high one.  The profile must still
    be the exact histogram."""
    import cpu_oracle as o
    n, S, turns = 50_000_000, 65536, 2
    ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), turns)
    rf = RFStation(ring, [4620], [0.0], [0.0])
    cl, cr = 0.0, 2.5e-9
    w = (cr - cl) / S
    rng = np.random.default_rng(7)
    k = rng.choice(3, size=n, p=[0.45, 0.45, 0.10])
    dt = np.where(k == 0, cl + 100.5 * w, cl + (100.5 + S // 2) * w)
    dt = np.where(k == 2, rng.uniform(cl, cr, n), dt)
    beam = Beam(ring, n, 1e11, dt=dt, dE=np.zeros(n))
    prof = Profile(beam, CutOptions(cut_left=cl, cut_right=cr, n_slices=S))
    fused = FusedTracker(RingAndRFTracker(rf, beam), prof, precision=precision)
    fused.track(turns)
    got = fused.profile_tensor().cpu().numpy()
    want = o.histogram(dt, cl, cr, S)
    assert got[100] > 2e7 and got[100 + S // 2] > 2e7
    np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(fused.dt.cpu().numpy(), dt)


@pytest.mark.parametrize("precision", ["f64", "f32p64"])
@pytest.mark.parametrize("chunks", [1, 3, 7])
def test_track_host_matches_device_tracking(cuda, precision, chunks):
    """Turns on page-locked host arrays, copied in and out every turn in
    chunks pipelined against the particle pass, give the device result bit
    for bit."""
    g = golden("track_full.npz")
    nt = int(g["n_turns"][0])
    out = []
    for host in (False, True):
        ring, rf, beam = build(g)
        prof = make_profile(g, beam)
        tiv = TotalInducedVoltage(beam, prof, impedance_objects("track_full.npz", beam, prof, rf))
        f = FusedTracker(RingAndRFTracker(rf, beam), prof, tiv, precision=precision)
        if host:
            hdt = f.dt.cpu().pin_memory()
            hdE = f.dE.cpu().pin_memory()
            f.track_host(hdt, hdE, nt - 1, chunks=chunks)
            f.track_host(hdt, hdE, 1, chunks=chunks)
            torch.cuda.synchronize()
            out.append((hdt.numpy().copy(), hdE.numpy().copy(),
                        f.profile_tensor().cpu().numpy()))
        else:
            f.track(nt)
            out.append((f.dt.cpu().numpy(), f.dE.cpu().numpy(),
                        f.profile_tensor().cpu().numpy()))
        assert rf.counter[0] == nt
    for a, b in zip(out[0], out[1]):
        np.testing.assert_array_equal(a, b)
    if precision == "f64":
        assert normwise(out[1][0], g["dt"]) < 1e-11
        np.testing.assert_array_equal(out[1][2], g["profiles"][-1])


@pytest.mark.parametrize("turns_per_graph", [1, 4])
@pytest.mark.parametrize("kernel", ["plain", "tma", "packed"])
def test_fused_interpolated_tracker_matches_reference(cuda, turns_per_graph, kernel):
    """RingAndRFTracker(interpolation=True) through the fused engine: the
    head interpolates RF voltage at the bin centres + induced voltage, the
    particle pass applies that one kick (tracker.py:586-601), against the
    reference objects' run (track_interp.npz)."""
    name = "track_interp.npz"
    g = golden(name)
    ring, rf, beam = build(g)
    prof = make_profile(g, beam)
    tiv = TotalInducedVoltage(beam, prof, impedance_objects(name, beam, prof, rf))
    tracker = RingAndRFTracker(rf, beam, solver=str(g["solver"][0]), interpolation=True,
                               profile=prof, total_induced_voltage=tiv)
    fused = FusedTracker(tracker, prof, tiv, precision="f64",
                         turns_per_graph=turns_per_graph, kernel=kernel)
    nt = int(g["n_turns"][0])
    fused.track(nt - 1)
    assert normwise(fused.induced_voltage_tensor().cpu().numpy(), g["vind"][nt - 2]) < 1e-10
    np.testing.assert_array_equal(fused.profile_tensor().cpu().numpy(), g["profiles"][nt - 1])
    fused.track(1)
    assert normwise(beam.dt.cpu().numpy(), g["dt"]) < 1e-11
    assert normwise(beam.dE.cpu().numpy(), g["dE"]) < 1e-11
    np.testing.assert_array_equal(fused.profile_tensor().cpu().numpy(), g["profiles"][-1])


@pytest.mark.parametrize("precision,kernel", [("f64", "auto"), ("q32p64", "auto"),
                                              ("f64", "packed"), ("q32p64", "packed")])
def test_fused_interpolated_tracker_without_impedance(cuda, precision, kernel):
    """Interpolated RF kick only (no induced voltage), double RF with an
    acceleration-free programme: the fused engine against the drop-in
    objects (bmath rf_volt_comp + linear_interp_kick, turn by turn)."""
    n, S, turns = 20001, 300, 6
    res = []
    for fused_path in (False, True):
        ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), turns)
        rf = RFStation(ring, [4620, 4 * 4620], [4.5e6, 0.45e6], [0.0, np.pi], n_rf=2)
        centre = (rf.phi_s[0] - rf.phi_rf[0, 0]) / rf.omega_rf[0, 0]
        from blond_b200.beam.distributions import bigaussian_arrays
        rng = np.random.default_rng(3)
        dt0 = centre + 0.5e-9 * rng.standard_normal(n)
        dE0 = 2e7 * rng.standard_normal(n)
        beam = Beam(ring, n, 1e10, dt=dt0, dE=dE0)
        prof = Profile(beam, CutOptions(cut_left=centre - 1.5e-9, cut_right=centre + 1.5e-9,
                                        n_slices=S))
        tracker = RingAndRFTracker(rf, beam, interpolation=True, profile=prof)
        if fused_path:
            f = FusedTracker(tracker, prof, precision=precision, turns_per_graph=4,
                             kernel=kernel)
            f.track(turns)
            f.sync()
        else:
            for _ in range(turns):
                tracker.track()
                prof.track()
        res.append((beam.dt.cpu().numpy(), beam.dE.cpu().numpy(),
                    prof.n_macroparticles.cpu().numpy()))
    (dt_a, dE_a, p_a), (dt_b, dE_b, p_b) = res
    tol = 1e-12 if precision == "f64" else 1e-8
    assert normwise(dt_b, dt_a) < tol
    assert normwise(dE_b, dE_a) < tol
    if precision == "f64":
        np.testing.assert_array_equal(p_b, p_a)
    else:
        assert np.abs(p_b - p_a).sum() <= 4


@pytest.mark.parametrize("kernel", ["plain", "tma"])
def test_fused_smooth_slicing_matches_reference(cuda, kernel):
    """Profile(smooth=True) through the fused engine: the slice_smooth
    weights (histogram.cpp:75-132, negative entries included) deposited in
    64-bit fixed point after every particle pass, the induced voltage of
    that profile, against the reference objects' run (track_smooth.npz):
    coordinates 1e-11, profiles and induced voltages 1e-10 normwise; two
    runs give the same bits."""
    name = "track_smooth.npz"
    g = golden(name)
    out = []
    for _ in range(2):
        ring, rf, beam = build(g)
        prof = make_profile(g, beam, smooth=True)
        tiv = TotalInducedVoltage(beam, prof, impedance_objects(name, beam, prof, rf))
        fused = FusedTracker(RingAndRFTracker(rf, beam, solver=str(g["solver"][0])), prof,
                             tiv, precision="f64", turns_per_graph=2, kernel=kernel)
        nt = int(g["n_turns"][0])
        assert normwise(fused.profile_tensor().cpu().numpy(), g["profiles"][0]) < 1e-10
        fused.track(nt - 1)
        assert normwise(fused.induced_voltage_tensor().cpu().numpy(), g["vind"][nt - 2]) < 1e-10
        fused.track(1)
        assert normwise(beam.dt.cpu().numpy(), g["dt"]) < 1e-11
        assert normwise(beam.dE.cpu().numpy(), g["dE"]) < 1e-11
        p = fused.profile_tensor().cpu().numpy()
        assert normwise(p, g["profiles"][-1]) < 1e-10
        assert p.min() < 0 or g["profiles"][-1].min() >= 0
        out.append((beam.dt.cpu().numpy(), p))
    for a, b in zip(*out):
        np.testing.assert_array_equal(a, b)
