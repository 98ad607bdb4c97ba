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
def test_fused_engine_matches_reference(cuda, name, turns_per_graph):
    g = golden(name)
    ring, rf, beam = build(g)
    prof = make_profile(g, beam)
    ivs = impedance_objects(name, beam, prof, rf)
    tiv = TotalInducedVoltage(beam, prof, ivs) if ivs else None
    tracker = RingAndRFTracker(rf, beam, solver=str(g["solver"][0]))
    fused = FusedTracker(tracker, prof, tiv, precision="f64",
                         turns_per_graph=turns_per_graph)
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
