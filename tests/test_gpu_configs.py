"""The benchmarked configurations against the oracle, at full size.

C2 -- the default bench line: 1e7 protons at 26 GeV/c, h = 4620, 4.5 MV,
2^14 slices over 2.5 ns, a broadband resonator (5 MOhm, 1 GHz, Q = 1)
through InducedVoltageFreq (n_fft 16384), intensity 1e10.  The tracker is
built by bench.build_fused itself (the autotuned launch shape, 50-turn
graphs), so the run checked here is the run the bench times.  Bars
(the reference's one-turn parity definitions): dt/dE within 1e-12
normwise, slice counts exact, induced voltage within 1e-10 normwise, over
3 turns (after each turn, from the oracle's state of the previous turn).
The precision form F32P64 is held to its own bar after the same turns:
rms bunch length and energy spread of the in-window particles within 1e-5
of the FP64 oracle, every particle counted once.

C1 -- the reference's CPU case: same ring and RF, 1e6 protons, 100 slices
over 2.5 ns, no impedance, FP64, 1000 turns.  Over 1000 turns the device
sine and the oracle's (glibc) may differ in the last bit for a few
arguments, and the synchrotron motion carries such a difference along
without amplifying it inside the bucket.  Bars after 1000 turns: dt/dE
within 1e-10 normwise; every slice count within 2 of the oracle's and the
counts' sum exact (a particle one rounding away from a bin edge may sit
on the other side).
"""
import numpy as np
import pytest
import torch

from conftest import normwise

pytestmark = pytest.mark.gpu


def _bench():
    import bench
    return bench


def _c2_oracle_turn(o, dt, dE, ring, rf, prof, iv, t):
    """One oracle turn of C2 from (dt, dE) at turn t: returns dt, dE, the
    final profile and the turn's induced voltage."""
    odt, odE, oprof, ov = o.track_oracle(
        dt, dE, ring, rf, (prof.cut_left, prof.cut_right), prof.bin_centers,
        int(prof.n_slices), 1, impedance=(iv.n_fft, iv.total_impedance.cpu().numpy()),
        intensity=1e10, start_turn=t)
    return odt, odE, oprof[-1], ov[-1]


def test_c2_fp64_matches_oracle_turn_by_turn(cuda):
    import cpu_oracle as o
    bench = _bench()
    turns = 3
    fused, beam, n_fft = bench.build_fused(int(1e7), 16384, turns, "f64")
    assert n_fft == 16384
    iv = fused.tiv.induced_voltage_list[0]
    ring, rf = bench.machine(turns)[0], fused.rf
    dt = beam.dt.cpu().numpy().copy()
    dE = beam.dE.cpu().numpy().copy()
    assert fused.autotune()["kernel"] in ("plain", "tma", "stab", "packed")
    for t in range(turns):
        fused.track(1)
        fused.check()
        dt, dE, oprof, ov = _c2_oracle_turn(o, dt, dE, ring, rf, fused.profile, iv, t)
        assert normwise(beam.dt.cpu().numpy(), dt) < 1e-12
        assert normwise(beam.dE.cpu().numpy(), dE) < 1e-12
        np.testing.assert_array_equal(fused.profile_tensor().cpu().numpy(), oprof)
        assert normwise(fused.induced_voltage_tensor().cpu().numpy(), ov) < 1e-10
        # continue from the device state, so every turn is a one-turn check
        dt = beam.dt.cpu().numpy().copy()
        dE = beam.dE.cpu().numpy().copy()


def test_c2_fp64_graph_replay_matches_oracle(cuda):
    """The bench's timed form: turns replayed from one captured graph."""
    import cpu_oracle as o
    bench = _bench()
    turns = 3
    fused, beam, _ = bench.build_fused(int(1e7), 16384, turns, "f64")
    fused.eng.call("tune", 0, 0, turns)  # one graph of all the turns
    iv = fused.tiv.induced_voltage_list[0]
    ring = bench.machine(turns)[0]
    dt0 = beam.dt.cpu().numpy().copy()
    dE0 = beam.dE.cpu().numpy().copy()
    fused.prepare()
    fused.track(turns)
    fused.check()
    odt, odE, oprof, ov = o.track_oracle(
        dt0, dE0, ring, fused.rf, (fused.profile.cut_left, fused.profile.cut_right),
        fused.profile.bin_centers, 16384, turns,
        impedance=(iv.n_fft, iv.total_impedance.cpu().numpy()), intensity=1e10)
    assert normwise(beam.dt.cpu().numpy(), odt) < 1e-12
    assert normwise(beam.dE.cpu().numpy(), odE) < 1e-12
    np.testing.assert_array_equal(fused.profile_tensor().cpu().numpy(), oprof[-1])
    assert normwise(fused.induced_voltage_tensor().cpu().numpy(), ov[-1]) < 1e-10


def test_c2_f32p64_bunch_statistics_vs_oracle(cuda):
    import cpu_oracle as o
    bench = _bench()
    turns = 3
    fused, beam, _ = bench.build_fused(int(1e7), 16384, turns, "f32p64")
    iv = fused.tiv.induced_voltage_list[0]
    ring = bench.machine(turns)[0]
    dt0 = beam.dt.cpu().numpy().copy()
    dE0 = beam.dE.cpu().numpy().copy()
    fused.track(turns)
    fused.sync()
    odt, odE, oprof, _ = o.track_oracle(
        dt0, dE0, ring, fused.rf, (fused.profile.cut_left, fused.profile.cut_right),
        fused.profile.bin_centers, 16384, turns,
        impedance=(iv.n_fft, iv.total_impedance.cpu().numpy()), intensity=1e10)
    dt, dE = beam.dt.cpu().numpy(), beam.dE.cpu().numpy()
    w = (odt > fused.profile.cut_left) & (odt < fused.profile.cut_right)
    for a, b in ((dt, odt), (dE, odE)):
        assert abs(np.std(a[w]) / np.std(b[w]) - 1) < 1e-5
    got = fused.profile_tensor().cpu().numpy()
    assert got.sum() == oprof[-1].sum()
    # float32 energies move a few particles across 0.15 ps bin edges
    assert np.abs(got - oprof[-1]).sum() <= 1e-3 * len(dt)


def test_c1_fp64_1000_turns_vs_oracle(cuda):
    import cpu_oracle as o
    from blond_b200.beam.beam import Beam
    from blond_b200.beam.profile import CutOptions, Profile
    from blond_b200.engine import FusedTracker
    from blond_b200.trackers.tracker import RingAndRFTracker
    bench = _bench()
    n, S, turns = 1_000_000, 100, 1000
    ring, rf = bench.machine(turns)
    dt0, dE0, centre = bench.host_bunch(ring, rf, n, 0)
    beam = Beam(ring, n, 1e10, dt=dt0, dE=dE0, dtype=torch.float64)
    cl, cr, _ = bench.window(centre, S)
    prof = Profile(beam, CutOptions(cut_left=cl, cut_right=cr, n_slices=S))
    fused = FusedTracker(RingAndRFTracker(rf, beam), prof, precision="f64")
    fused.track(turns)
    fused.check()
    odt, odE, oprof, _ = o.track_oracle(dt0, dE0, ring, rf, (cl, cr), prof.bin_centers, S,
                                        turns)
    ed, eE = normwise(beam.dt.cpu().numpy(), odt), normwise(beam.dE.cpu().numpy(), odE)
    got = fused.profile_tensor().cpu().numpy()
    print(f"C1 after {turns} turns: dt {ed:.2e}, dE {eE:.2e}, "
          f"max count difference {np.abs(got - oprof[-1]).max():.0f}")
    assert ed < 1e-10 and eE < 1e-10
    assert got.sum() == oprof[-1].sum()
    assert np.abs(got - oprof[-1]).max() <= 2
