"""Beam statistics and the monitors on the device.

* blond_beam_statistics against numpy's mean / std / dot over the particles
  with id != 0 (Beam.statistics, beam/beam.py:430-458): float64 within
  1e-13 relative, float32 coordinates within 1e-6 (numpy sums float32
  pairwise, the kernel in float64).
* BunchMonitor (monitors.py:36-466) over a tracked bunch with a beam-phase
  loop and an rms profile fit, flushed every 10 turns: every row of every
  dataset against values taken on the host turn by turn.
* SlicesMonitor (monitors.py:470-508): every turn's profile column.
"""
import os

import numpy as np
import pytest
import torch

from blond_b200 import bmath as bm
from blond_b200.beam.beam import Beam, Proton
from blond_b200.beam.distributions import bigaussian
from blond_b200.beam.profile import CutOptions, FitOptions, Profile
from blond_b200.input_parameters.rf_parameters import RFStation
from blond_b200.input_parameters.ring import Ring
from blond_b200.llrf.beam_feedback import BeamFeedback
from blond_b200.monitors.monitors import BunchMonitor, SlicesMonitor
from blond_b200.trackers.tracker import RingAndRFTracker

pytestmark = pytest.mark.gpu


def host_stats(dt, dE, id=None):
    dt, dE = np.asarray(dt, np.float64), np.asarray(dE, np.float64)
    if id is not None:
        keep = np.asarray(id) != 0
        dt, dE = dt[keep], dE[keep]
    return np.array([dt.size, dt.mean(), dt.std(), dE.mean(), dE.std(),
                     np.pi * dE.std() * dt.std(), dt @ dt, dE @ dE])


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_statistics_match_numpy(cuda, dtype):
    rng = np.random.default_rng(3)
    n = 1_000_003
    dt = 2.5e-9 + 0.3e-9 * rng.normal(size=n)
    dE = 1e7 * rng.normal(size=n) + 3e5
    id = np.arange(1, n + 1)
    id[rng.choice(n, 5000, replace=False)] = 0
    tdt = torch.as_tensor(dt, device="cuda").to(dtype)
    tdE = torch.as_tensor(dE, device="cuda").to(dtype)
    want = host_stats(tdt.cpu().numpy(), tdE.cpu().numpy(), id)
    out = None
    for _ in range(2):  # the second call shifts by the first call's means
        out = bm.beam_statistics(tdt, tdE, torch.as_tensor(id, device="cuda"), out=out)
        got = out.cpu().numpy()
        rtol = 1e-13 if dtype == torch.float64 else 1e-6
        assert got[0] == want[0]
        np.testing.assert_allclose(got[1:], want[1:], rtol=rtol)
    got = bm.beam_statistics(tdt, tdE).cpu().numpy()  # everyone alive
    np.testing.assert_allclose(got, host_stats(tdt.cpu().numpy(), tdE.cpu().numpy()),
                               rtol=1e-13 if dtype == torch.float64 else 1e-6)


def machine(n_turns):
    ring = Ring(6911.5038, 1.0 / 17.95142852 ** 2, 25.92e9, Proton(), n_turns)
    rf = RFStation(ring, 4620, 4.5e6, 0)
    beam = Beam(ring, 100000, 1e10)
    bigaussian(ring, rf, beam, 0.2e-9, seed=11)
    beam.dt += 0.1e-9
    return ring, rf, beam


def test_beam_statistics_attributes(cuda):
    ring, rf, beam = machine(5)
    beam.statistics()
    want = host_stats(beam.dt.cpu().numpy(), beam.dE.cpu().numpy())
    np.testing.assert_allclose([beam.mean_dt, beam.sigma_dt, beam.mean_dE, beam.sigma_dE,
                                beam.epsn_rms_l], want[1:6], rtol=1e-13)
    beam.sigma_dt = 1.0  # attributes stay assignable, as in the reference
    assert beam.sigma_dt == 1.0


def load(filename):
    if os.path.exists(filename + ".npz"):
        return dict(np.load(filename + ".npz"))
    import h5py
    with h5py.File(filename + ".h5", "r") as f:
        g = f[list(f.keys())[0]]
        return {k: g[k][()] for k in g}


def test_bunch_monitor_rows(cuda, tmp_path):
    T = 30
    ring, rf, beam = machine(T)
    profile = Profile(beam, CutOptions(cut_left=0, cut_right=rf.t_rf[0, 0], n_slices=256),
                      FitOptions(fit_option="rms"))
    loop = BeamFeedback(ring, rf, profile, {"machine": "LHC_F", "PL_gain": 1000.0,
                                            "FL_gain": 0.05})
    tracker = RingAndRFTracker(rf, beam, profile=profile, beam_feedback=loop)
    fn = str(tmp_path / "out" / "bunch")
    mon = BunchMonitor(ring, rf, beam, fn, buffer_time=10, profile=profile, phase_loop=loop)
    rows = [host_stats(beam.dt.cpu().numpy(), beam.dE.cpu().numpy())]
    extra = [(profile.bunchLength, rf.omega_rf[0, 0], loop.phi_beam)]
    for turn in range(T - 1):  # the monitor's first row came at construction
        profile.track()
        tracker.track()
        mon.track()
        rows.append(host_stats(beam.dt.cpu().numpy(), beam.dE.cpu().numpy()))
        extra.append((profile.bunchLength, rf.omega_rf[0, turn + 1], loop.phi_beam))
    d = load(fn)
    rows = np.array(rows)
    assert d["mean_dt"].shape == (T + 1,) and d["mean_dt"].dtype == np.float32
    for name, k in (("n_macroparticles_alive", 0), ("mean_dt", 1), ("sigma_dt", 2),
                    ("mean_dE", 3), ("sigma_dE", 4), ("epsn_rms_l", 5)):
        np.testing.assert_allclose(d[name][:T], rows[:, k].astype(np.float32), rtol=1e-6)
    extra = np.array(extra)
    np.testing.assert_allclose(d["bunch_length"][:T], extra[:, 0].astype(np.float32), rtol=1e-6)
    np.testing.assert_array_equal(d["PL_omegaRF"][:T], extra[:, 1])
    np.testing.assert_allclose(d["PL_bunch_phase"][:T], extra[:, 2].astype(np.float32),
                               rtol=1e-6)
    assert np.all(d["mean_dt"][T:] == 0)  # the last row is not flushed yet


def test_slices_monitor(cuda, tmp_path):
    ring, rf, beam = machine(20)
    profile = Profile(beam, CutOptions(cut_left=0, cut_right=rf.t_rf[0, 0], n_slices=128))
    tracker = RingAndRFTracker(rf, beam)
    fn = str(tmp_path / "slices")
    mon = SlicesMonitor(fn, 20, profile, buffer_size=8)
    want = []
    for _ in range(20):
        tracker.track()
        profile.track()
        mon.track()
        want.append(profile.n_macroparticles.cpu().numpy())
    mon.close()
    d = load(fn)
    np.testing.assert_array_equal(d["n_macroparticles"], np.array(want, np.float32).T)
