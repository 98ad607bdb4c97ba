"""The beam-phase loop on the device vs the reference.

* blond_beam_phase / blond_beam_phase_fast (both precisions) against the
  reference's compiled beam_phase.cpp outputs (tests/golden/beam_phase.npz).
* BeamFeedback for every machine type ('LHC' with and without the synchro
  loop and window, 'LHC_F', 'SPS_F' with and without the sharp window,
  'SPS_RL', 'PSB') tracked for 200 turns through RingAndRFTracker /
  FullRingAndRF, against the reference objects on the same bunch
  (tests/golden/beam_feedback.npz; the SPS set-up of the reference's
  unittests/llrf/test_beam_feedback.py:22-59).  Bars: the loop's per-turn
  beam phase, phase error and frequency correction within 1e-9 normwise,
  the RF frequency and phase programmes within 1e-12, coordinates 1e-9.
* The same loops inside the fused engine's turn (FusedTracker; the beam
  phase, loop filter and RF programme correction run on the device, inside
  the head kernel when there is an FFT impedance and in an all-SM pass
  otherwise), at the same bars, tracked both turn by turn and 200 turns in
  one call; fused.sync() brings the loop state back to the host objects.
"""
import numpy as np
import pytest
import torch

from conftest import golden, normwise
from blond_b200 import bmath as bm
from blond_b200.beam.beam import Beam, Proton
from blond_b200.beam.distributions import bigaussian
from blond_b200.beam.profile import CutOptions, Profile
from blond_b200.engine import FusedTracker
from blond_b200.impedances.impedance import InducedVoltageFreq, TotalInducedVoltage
from blond_b200.impedances.impedance_sources import Resonators
from blond_b200.input_parameters.rf_parameters import RFStation
from blond_b200.input_parameters.ring import Ring
from blond_b200.llrf.beam_feedback import BeamFeedback
from blond_b200.trackers.tracker import FullRingAndRF, RingAndRFTracker

pytestmark = pytest.mark.gpu

CASES = {
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
    # with a broadband resonator: the fused engine runs the loop inside its
    # spectral head kernel
    "LHC_F_Z": ("sps", {"machine": "LHC_F", "PL_gain": 1000.0, "FL_gain": 0.05}, 0),
    "SPS_RL_Z": ("sps", {"machine": "SPS_RL", "PL_gain": 1000.0, "RL_gain": 1e6,
                         "sample_dE": 2}, 0),
}
IMPEDANCE = {"LHC_F_Z", "SPS_RL_Z"}


def setup_case(name):
    kind, cfg, delay = CASES[name]
    cfg = {k: (list(v) if isinstance(v, list) else v) for k, v in cfg.items()}
    ring, rf, sigma, shift = machine(kind)
    beam = Beam(ring, 200000, 1e11 if name in IMPEDANCE else 1.2e6)
    bigaussian(ring, rf, beam, sigma, seed=1234)
    beam.dt += shift
    profile = Profile(beam, CutOptions(cut_left=0, cut_right=rf.t_rf[0, 0], n_slices=1024))
    loop = BeamFeedback(ring, rf, profile, cfg, delay=delay)
    tracker = RingAndRFTracker(rf, beam, profile=profile, beam_feedback=loop)
    tiv = None
    if name in IMPEDANCE:
        tiv = TotalInducedVoltage(beam, profile, [InducedVoltageFreq(
            beam, profile, [Resonators(5e6, 1e9, 1.0)])])
    return rf, beam, profile, loop, tracker, tiv


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_beam_phase_kernels_match_reference(cuda, dtype):
    g = golden("beam_phase.npz")
    tag = "f64" if dtype == torch.float64 else "f32"
    rtol = 1e-13 if tag == "f64" else 1e-4
    for k, (want_w, want_f) in enumerate(g[f"{tag}_coeff"]):
        bc = torch.as_tensor(g[f"{tag}_{k}_bc"], device="cuda")
        p = torch.as_tensor(g[f"{tag}_{k}_profile"], device="cuda")
        alpha, om, ph, bs = g[f"{tag}_{k}_params"]
        np.testing.assert_allclose(bm.beam_phase(bc, p, alpha, om, ph, bs), want_w, rtol=rtol)
        np.testing.assert_allclose(bm.beam_phase_fast(bc, p, om, ph, bs), want_f, rtol=rtol)
        dev = bm.beam_phase(bc, p, alpha, om, ph, bs, device_result=True)
        assert isinstance(dev, torch.Tensor) and dev.dtype == dtype
    # a sub-range is the reference's call on the sliced arrays; empty gives NaN
    bc = torch.as_tensor(g["f64_0_bc"], device="cuda")
    p = torch.as_tensor(g["f64_0_profile"], device="cuda")
    alpha, om, ph, bs = g["f64_0_params"]
    a = bm.beam_phase(bc, p, alpha, om, ph, bs, start=300, stop=700)
    b = bm.beam_phase(bc[300:700].clone(), p[300:700].clone(), alpha, om, ph, bs)
    assert a == b
    assert np.isnan(bm.beam_phase(bc, p, alpha, om, ph, bs, start=5, stop=5))


def machine(kind, n_turns=200):
    if kind == "sps":
        ring = Ring(6911.5038, 1.0 / 17.95142852 ** 2, 25.92e9, Proton(), n_turns)
        rf = RFStation(ring, 4620, 4.5e6, 0)
        return ring, rf, 0.05e-9, 0.1e-9
    ring = Ring(26658.883, 3.225e-4, 450e9, Proton(), n_turns)
    rf = RFStation(ring, 35640, 6e6, 0)
    return ring, rf, 0.25e-9, 0.2e-9


@pytest.mark.parametrize("name", list(CASES))
def test_beam_feedback_tracks_reference(cuda, name):
    g = golden("beam_feedback.npz")
    rf, beam, profile, loop, section, tiv = setup_case(name)
    tracker = FullRingAndRF([section])
    trace = np.zeros((200, 4))
    for turn in range(200):
        trace[turn, 0] = float(beam.dt.mean())
        if tiv is not None:
            tiv.track()
            tracker.track()
            profile.track()
        else:
            profile.track()
            tracker.track()
        trace[turn, 1:] = (loop.phi_beam, loop.dphi, loop.domega_rf)
    want = g[f"{name}_trace"]
    for col in range(4):
        assert normwise(trace[:, col], want[:, col]) < 1e-9, (name, col)
    assert normwise(rf.omega_rf[0], g[f"{name}_omega_rf"]) < 1e-12
    assert normwise(rf.phi_rf[0], g[f"{name}_phi_rf"]) < 1e-12
    assert normwise(beam.dt.cpu().numpy()[::997], g[f"{name}_dt"]) < 1e-9
    assert normwise(beam.dE.cpu().numpy()[::997], g[f"{name}_dE"]) < 1e-9




@pytest.mark.parametrize("name", list(CASES))
def test_fused_beam_feedback_matches_reference(cuda, name):
    g = golden("beam_feedback.npz")
    rf, beam, profile, loop, tracker, tiv = setup_case(name)
    fused = FusedTracker(tracker, profile, tiv, precision="f64")
    want = g[f"{name}_trace"]
    if name in ("LHC", "PSB", "SPS_RL_Z"):
        # turn by turn: the loop state round-trips through the host objects
        mean_dt = np.zeros(200)
        trace = np.zeros((200, 3))
        for turn in range(200):
            mean_dt[turn] = float(beam.dt.mean())
            fused.track(1)
            fused.sync()
            trace[turn] = (loop.phi_beam, loop.dphi, loop.domega_rf)
        assert normwise(mean_dt, want[:, 0]) < 1e-9
    else:
        fused.track(200)
        fused.sync()
        trace = fused.loop_trace[:200]
        assert (loop.phi_beam, loop.dphi, loop.domega_rf) == tuple(trace[-1])
    for col in range(3):
        assert normwise(trace[:, col], want[:, col + 1]) < 1e-9, (name, col)
    assert normwise(rf.omega_rf[0], g[f"{name}_omega_rf"]) < 1e-12
    assert normwise(rf.phi_rf[0], g[f"{name}_phi_rf"]) < 1e-12
    assert rf.counter[0] == 200
    assert normwise(beam.dt.cpu().numpy()[::997], g[f"{name}_dt"]) < 1e-9
    assert normwise(beam.dE.cpu().numpy()[::997], g[f"{name}_dE"]) < 1e-9


def test_fused_beam_feedback_f32p64_follows_f64(cuda):
    """F32P64 kick arithmetic under the same loop: the frequency offsets it
    produces stay finite and within 1e-3 (normwise) of the FP64 ones over
    200 turns."""
    out = {}
    for prec in ("f64", "f32p64"):
        rf, beam, profile, loop, tracker, _ = setup_case("LHC_F")
        fused = FusedTracker(tracker, profile, None, precision=prec)
        fused.track(200)
        fused.sync()
        out[prec] = rf.omega_rf[0].copy() - rf.omega_rf_d[0]
    assert np.all(np.isfinite(out["f32p64"]))
    assert normwise(out["f32p64"], out["f64"]) < 1e-3
