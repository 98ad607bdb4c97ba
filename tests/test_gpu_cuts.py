"""The automatic slicing frame on the device (blond_cut_limits) against the
reference's CutOptions.set_cuts (beam/profile.py:175-211), fixtures from
tests/golden/gen_golden.py (cut_options.npz, profile_golden.npz).

Bars: the default frame (min/max -/+ 5 % of the spread) bit for bit, so
the bin centres and the profile counts are the reference's exactly; the
n_sigma frame (numpy mean and std) within a few ulps; the 'rad' frame and
its counts exactly.
"""
import numpy as np
import pytest
import torch

from conftest import golden
from blond_b200 import bmath as bm
from blond_b200.beam.beam import Beam, Proton
from blond_b200.beam.profile import CutOptions, Profile
from blond_b200.input_parameters.rf_parameters import RFStation
from blond_b200.input_parameters.ring import Ring

pytestmark = pytest.mark.gpu

CASES = [("default", None), ("nsigma3", 3), ("nsigma55", 5.5)]


def _dt(name):
    if name == "unit":
        return golden("profile_golden.npz")["dt"]
    return golden("cut_options.npz")["dt_bunch"]


@pytest.mark.parametrize("name", ["unit", "bunch"])
@pytest.mark.parametrize("tag,n_sigma", CASES)
def test_cut_limits_match_the_reference(cuda, name, tag, n_sigma):
    g = golden("cut_options.npz")
    dt = _dt(name)
    want = g[f"{name}_{tag}"]
    got = bm.cut_limits(torch.tensor(dt, device="cuda"), n_sigma).cpu().numpy()
    ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), 10)
    beam = Beam(ring, len(dt), 1e10, dt=dt, dE=np.zeros(len(dt)))
    prof = Profile(beam, CutOptions(n_slices=64, n_sigma=n_sigma))
    if n_sigma is None:
        np.testing.assert_array_equal(got, want)
        np.testing.assert_array_equal(prof.bin_centers, g[f"{name}_{tag}_bc"])
    else:
        assert np.max(np.abs(got - want)) <= 4 * np.spacing(np.max(np.abs(want)))
        np.testing.assert_allclose(prof.bin_centers, g[f"{name}_{tag}_bc"], rtol=1e-14)


def test_default_and_rad_frames_give_the_reference_profiles(cuda):
    """The reference's own profile unit test (test_beam_profile_object.py:
    169-204): the default frame and 200 slices over 0..2 pi rad, counts
    exact."""
    g = golden("profile_golden.npz")
    dt = g["dt"]
    ring = Ring(125, 0.001, 1e9, Proton(), 1)
    rf = RFStation(ring, [1], [7e6], [0.0])
    beam = Beam(ring, len(dt), 1e10, dt=dt, dE=np.zeros(len(dt)))
    p1 = Profile(beam)
    p1.track()
    np.testing.assert_array_equal([p1.cut_left, p1.cut_right], g["cuts1"])
    np.testing.assert_array_equal(p1.n_macroparticles.cpu().numpy(), g["counts1"])
    p2 = Profile(beam, CutOptions(cut_left=0, cut_right=2 * np.pi, n_slices=200,
                                  cuts_unit="rad", rf_station=rf))
    p2.track()
    np.testing.assert_array_equal([p2.cut_left, p2.cut_right], g["cuts2"])
    np.testing.assert_array_equal(p2.n_macroparticles.cpu().numpy(), g["counts2"])


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_cut_limits_over_many_blocks_and_nan(cuda, dtype):
    """1e7 values (every block's partial, then the last block's combine):
    exactly numpy's frame; a NaN anywhere gives NaN cuts, as numpy."""
    rng = np.random.default_rng(5)
    x = rng.normal(3e-9, 4e-10, 10_000_001).astype(np.float64 if dtype == torch.float64
                                                    else np.float32)
    t = torch.tensor(x, device="cuda")
    lo, hi = float(x.min()), float(x.max())
    want = [lo - 0.05 * (hi - lo), hi + 0.05 * (hi - lo)]
    np.testing.assert_array_equal(bm.cut_limits(t).cpu().numpy(), want)
    m, s = np.mean(x.astype(np.float64)), np.std(x.astype(np.float64))
    got = bm.cut_limits(t, 4).cpu().numpy()
    np.testing.assert_allclose(got, [m - 2 * s, m + 2 * s], rtol=1e-14)
    t[7_777_777] = float("nan")
    assert np.isnan(bm.cut_limits(t).cpu().numpy()).all()
