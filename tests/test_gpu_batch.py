"""Batched beams (blond_batch_*): each beam of a heterogeneous batch --
ragged particle counts (one particle, chunk tails, several chunks), its own
double-RF voltage, bunch length, slicing window and three resonators --
against the CPU oracle and against the single-beam engine.

Bars (FP64): coordinates within 1e-12 of the bunch scale, slice counts
exact, induced voltage within 1e-10 normwise; the batch reproduces the
single-beam engine bit for bit.  F32P64: rms bunch length and energy
spread within 1e-5 of FP64 after 100 turns.
"""
import numpy as np
import pytest
import torch

import cpu_oracle as o
from conftest import normwise
from blond_b200.batch import BatchTracker
from blond_b200.beam.beam import Beam, Proton
from blond_b200.beam.distributions import _get_dE_from_dt, bigaussian_arrays
from blond_b200.beam.profile import CutOptions, Profile
from blond_b200.engine import FusedTracker
from blond_b200.impedances.impedance import InducedVoltageFreq, TotalInducedVoltage
from blond_b200.impedances.impedance_sources import Resonators
from blond_b200.input_parameters.rf_parameters import RFStation
from blond_b200.input_parameters.ring import Ring
from blond_b200.trackers.tracker import RingAndRFTracker

pytestmark = pytest.mark.gpu

S = 512
COUNTS = [3000, 1, 32768 * 2 + 5, 777, 40001]


def make_beam(k, n, turns, S=S):
    """Beam k of a double-RF scan (h, 4h, V2/V1 = 0.1, phi2 = pi)."""
    rng = np.random.default_rng(100 + k)
    V1 = 2e6 + 5e6 * rng.random()
    ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), turns)
    rf = RFStation(ring, [4620, 4 * 4620], [V1, 0.1 * V1], [0.0, np.pi], n_rf=2)
    centre = (rf.phi_s[0] - rf.phi_rf[0, 0]) / rf.omega_rf[0, 0]
    sdt = 0.2e-9 + 0.3e-9 * rng.random()
    dt, dE = bigaussian_arrays(n, sdt, _get_dE_from_dt(ring, rf, sdt), centre, k)
    beam = Beam(ring, n, 2e6 * n, dt=dt, dE=dE)
    prof = Profile(beam, CutOptions(cut_left=centre - 1.25e-9, cut_right=centre + 1.25e-9,
                                    n_slices=S))
    Q = np.exp(np.log(100) + (np.log(30000) - np.log(100)) * rng.random(3))
    iv = InducedVoltageFreq(beam, prof, [Resonators([2e5, 1e5, 5e4],
                                                    [200e6, 800e6, 1.4e9], Q)])
    tiv = TotalInducedVoltage(beam, prof, [iv])
    return ring, rf, beam, prof, tiv, iv, (dt, dE)


@pytest.mark.parametrize("S", [512, 4096])
def test_batch_matches_oracle_and_single_beam_engine(cuda, S):
    """512 slices: each chunk copies its beam's table into shared memory;
    4096: the table is gathered from global memory."""
    turns = 5
    built = [make_beam(k, n, turns, S) for k, n in enumerate(COUNTS)]
    batch = BatchTracker([(RingAndRFTracker(rf, beam), prof, tiv)
                          for _, rf, beam, prof, tiv, _, _ in built],
                         precision="f64", turns_per_graph=2)
    batch.track(turns)
    prof = batch.profiles_tensor().cpu().numpy()
    vind = batch.induced_voltages_tensor().cpu().numpy()
    for b, (ring, rf, beam, p, tiv, iv, (dt0, dE0)) in enumerate(built):
        odt, odE, oprof, ovind = o.track_oracle(
            dt0, dE0, ring, rf, (p.cut_left, p.cut_right), p.bin_centers, S, turns,
            impedance=(iv.n_fft, iv.total_impedance.cpu().numpy()),
            intensity=2e6 * len(dt0))
        dt, dE = (x.cpu().numpy() for x in batch.coordinates(b))
        assert np.max(np.abs(dt - odt)) / max(np.max(np.abs(odt)), 1e-9) < 1e-12, b
        assert np.max(np.abs(dE - odE)) / max(np.max(np.abs(odE)), 2e7) < 1e-12, b
        np.testing.assert_array_equal(prof[b], oprof[-1])
        assert normwise(vind[b], ovind[-1]) < 1e-10
    # the same beams one by one through the single-beam engine
    for b, n in enumerate(COUNTS):
        ring, rf, beam, p, tiv, iv, _ = make_beam(b, n, turns, S)
        f = FusedTracker(RingAndRFTracker(rf, beam), p, tiv, precision="f64",
                         turns_per_graph=2)
        f.track(turns)
        dt, dE = (x.cpu().numpy() for x in batch.coordinates(b))
        np.testing.assert_array_equal(dt, beam.dt.cpu().numpy())
        np.testing.assert_array_equal(dE, beam.dE.cpu().numpy())


@pytest.mark.parametrize("precision", ["f64", "q32p64"])
def test_batch_chunks_claimed_beyond_the_first_wave(cuda, precision):
    """More chunks than resident blocks (1024-particle chunks, one 256-thread
    block per SM): blocks claim chunks as they finish, largest first, across
    turns; every beam, chunk starts at odd offsets included, ends bit for
    bit where the single-beam engine leaves it."""
    turns = 4
    counts = [3000, 1, 200001, 777, 40001]
    # one energy unit for every beam (the default, from each beam's largest
    # |dE|, is too fine for the one-particle beam's energy swing)
    unit = {"energy_unit": 0.5} if precision == "q32p64" else {}
    built = [make_beam(k, n, turns) for k, n in enumerate(counts)]
    batch = BatchTracker([(RingAndRFTracker(rf, beam), prof, tiv)
                          for _, rf, beam, prof, tiv, _, _ in built],
                         precision=precision, turns_per_graph=2,
                         energy_units=[0.5] * len(counts) if unit else None)
    batch.set_shape(256, 1, 4, 1024, False)
    n_chunks = sum(-(-n // 1024) for n in counts)
    assert n_chunks > torch.cuda.get_device_properties(0).multi_processor_count
    batch.track(turns)
    batch.check()
    prof = batch.profiles_tensor().cpu().numpy()
    for b, n in enumerate(counts):
        ring, rf, beam, p, tiv, iv, _ = make_beam(b, n, turns)
        f = FusedTracker(RingAndRFTracker(rf, beam), p, tiv, precision=precision,
                         turns_per_graph=2, **unit)
        f.track(turns)
        dt, dE = (x.cpu().numpy() for x in batch.coordinates(b))
        np.testing.assert_array_equal(dt, f.dt.cpu().numpy())
        np.testing.assert_array_equal(dE, f.dE.cpu().numpy())
        np.testing.assert_array_equal(prof[b], f.profile_tensor().cpu().numpy())


def test_batch_f32p64_bunch_statistics(cuda):
    turns = 100
    counts = [20000, 50000, 30000]
    f64 = [make_beam(k, n, turns) for k, n in enumerate(counts)]
    f32 = [make_beam(k, n, turns) for k, n in enumerate(counts)]
    a = BatchTracker([(RingAndRFTracker(rf, b), p, t) for _, rf, b, p, t, _, _ in f64],
                     precision="f64")
    c = BatchTracker([(RingAndRFTracker(rf, b), p, t) for _, rf, b, p, t, _, _ in f32],
                     precision="f32p64")
    a.track(turns)
    c.track(turns)
    for b in range(len(counts)):
        x = [t.cpu().double().numpy() for t in a.coordinates(b)]
        y = [t.cpu().double().numpy() for t in c.coordinates(b)]
        p = f64[b][3]
        w = (x[0] > p.cut_left) & (x[0] < p.cut_right)
        for u, v in zip(x, y):
            assert abs(np.std(v[w]) / np.std(u[w]) - 1) < 1e-5


def test_batch_sync_writes_back_into_the_objects(cuda):
    built = [make_beam(k, n, 3) for k, n in enumerate([1000, 2000])]
    batch = BatchTracker([(RingAndRFTracker(rf, beam), prof, tiv)
                          for _, rf, beam, prof, tiv, _, _ in built], precision="f64")
    batch.track(3)
    batch.sync()
    for b, (_, rf, beam, prof, tiv, _, _) in enumerate(built):
        np.testing.assert_array_equal(beam.dt.cpu().numpy(),
                                      batch.coordinates(b)[0].cpu().numpy())
        assert rf.counter[0] == 3
        assert float(prof.n_macroparticles.sum()) <= beam.n_macroparticles


def test_batch_rejects_mixed_slice_counts(cuda):
    ring, rf, beam, prof, tiv, _, _ = make_beam(0, 100, 2)
    ring2 = Ring(6911.5, 1 / 18**2, 26e9, Proton(), 2)
    rf2 = RFStation(ring2, [4620, 4 * 4620], [4e6, 4e5], [0.0, np.pi], n_rf=2)
    beam2 = Beam(ring2, 100, 2e8, dt=beam.dt.cpu().numpy(), dE=beam.dE.cpu().numpy())
    prof2 = Profile(beam2, CutOptions(cut_left=prof.cut_left, cut_right=prof.cut_right,
                                      n_slices=256))
    with pytest.raises(ValueError):
        BatchTracker([(RingAndRFTracker(rf, beam), prof, None),
                      (RingAndRFTracker(rf2, beam2), prof2, None)])
