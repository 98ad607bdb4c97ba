"""Host-side logic of the drop-in layer against the reference (no GPU)."""
import numpy as np
import pytest

from conftest import golden, normwise
from blond_b200.beam.beam import Proton
from blond_b200.beam.distributions import _get_dE_from_dt, bigaussian_arrays
from blond_b200.impedances.impedance import induced_voltage_lengths
from blond_b200.input_parameters.rf_parameters import RFStation
from blond_b200.input_parameters.ring import Ring
from blond_b200.toolbox.next_regular import next_regular


def test_next_regular_table():
    g = golden("nfft_known.npz")
    got = np.array([next_regular(int(t)) for t in g["next_regular_targets"]])
    np.testing.assert_array_equal(got, g["next_regular_values"])


def test_n_fft_known_answers():
    """unittests/impedances/test_impedance.py:30-125 (16 slices over 5 ns)."""
    g = golden("nfft_known.npz")
    S, cl, cr = 16, 0.0, 5e-9
    bs = (cr - cl) / S
    n_iv, _ = induced_voltage_lengths(S, bs, cl, cr)
    assert [next_regular(n_iv), n_iv] == list(g["freq_default"])
    n_iv, _ = induced_voltage_lengths(S, bs, cl, cr, frequency_resolution=3e6)
    assert [next_regular(n_iv), n_iv] == list(g["freq_res3e6"]) == [1080, 1067]
    n_iv, _ = induced_voltage_lengths(S, bs, cl, cr)
    assert [next_regular(n_iv + S - 1), n_iv] == list(g["time_default"])
    n_iv, _ = induced_voltage_lengths(S, bs, cl, cr, wake_length=11e-9)
    assert [next_regular(n_iv + S - 1), n_iv] == list(g["time_wake11ns"])


def test_ring_and_rfstation_match_reference():
    g = golden("machine_c1.npz")
    ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), 1000)
    rf = RFStation(ring, [4620], [4.5e6], [0.0])
    for k in ("beta", "gamma", "energy", "momentum", "eta_0", "eta_1", "eta_2"):
        np.testing.assert_allclose(getattr(ring, k)[0, :3], g[k], rtol=1e-15, atol=0)
    np.testing.assert_allclose(ring.t_rev[:3], g["t_rev"], rtol=1e-15)
    np.testing.assert_allclose(rf.omega_rf[:, :3], g["omega_rf"], rtol=1e-15)
    np.testing.assert_allclose(rf.phi_s[:3], g["phi_s"], rtol=1e-15)
    np.testing.assert_allclose(rf.Q_s[:3], g["Q_s"], rtol=1e-14)
    np.testing.assert_allclose(rf.t_rf[:, :3], g["t_rf"], rtol=1e-15)
    rf2 = RFStation(Ring(6911.5, 1 / 18**2, 26e9, Proton(), 100),
                    [4620, 4 * 4620], [4.5e6, 0.45e6], [0.0, np.pi], n_rf=2)
    np.testing.assert_allclose(rf2.omega_rf[:, :3], g["omega_rf_2"], rtol=1e-15)


def test_bigaussian_streams_match_reference():
    g = golden("machine_c1.npz")
    ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), 1000)
    rf = RFStation(ring, [4620], [4.5e6], [0.0])
    sigma_dE = _get_dE_from_dt(ring, rf, 0.4e-9)
    assert np.isclose(sigma_dE, g["sigma_dE"][0], rtol=1e-15)
    centre = (rf.phi_s[0] - rf.phi_rf[0, 0]) / rf.omega_rf[0, 0]
    dt, dE = bigaussian_arrays(len(g["dt"]), 0.4e-9, sigma_dE, centre, 0)
    np.testing.assert_array_equal(dt, g["dt"])
    np.testing.assert_array_equal(dE, g["dE"])


def test_spectral_plan_factorisation_covers_next_regular_lengths():
    """Every even n_fft that next_regular can return up to 2^17 has M = n/2
    5-smooth, so the cluster transform takes it without the DFT path."""
    for t in range(7, 131073, 97):
        n = next_regular(t)
        if n > 131072:
            continue
        assert n % 2 == 0
        m = n // 2
        for f in (2, 3, 5):
            while m % f == 0:
                m //= f
        assert m == 1, n


def test_normwise_helper():
    assert normwise([1.0, 2.0], [1.0, 2.0]) == 0.0
    assert np.isclose(normwise([1.0, 2.2], [1.0, 2.0]), 0.1)


def test_bench_clock_sampler_reads_nvml(monkeypatch):
    """bench.py's clock record through a fake NVML: polled samples, the
    median SM clock, and the reasons decoded from the event-reason bits."""
    import os
    import sys
    import time
    import types
    fake = types.ModuleType("pynvml")
    fake.NVML_CLOCK_SM = 1
    fake.nvmlClocksEventReasonHwSlowdown = 0x8
    fake.nvmlClocksEventReasonHwThermalSlowdown = 0x40
    fake.nvmlClocksEventReasonSwThermalSlowdown = 0x20
    fake.nvmlClocksEventReasonSwPowerCap = 0x4
    fake.nvmlInit = lambda: None
    def by_uuid(u):
        raise RuntimeError("no such GPU")
    fake.nvmlDeviceGetHandleByUUID = by_uuid
    fake.nvmlDeviceGetHandleByIndex = lambda i: ("gpu", i)
    fake.nvmlDeviceGetMaxClockInfo = lambda h, c: 1965
    fake.nvmlDeviceGetClockInfo = lambda h, c: 1800
    fake.nvmlDeviceGetCurrentClocksEventReasons = lambda h: 0x4 | 0x1
    monkeypatch.setitem(sys.modules, "pynvml", fake)
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    c = bench.ClockSampler(0)
    time.sleep(0.02)
    r = c.stop()
    assert r["samples"] >= 3
    assert r["sm_mhz"] == 1800.0 and r["sm_max_mhz"] == 1965.0
    assert r["reasons"] == ["sw_power_cap"]
    assert r["source"].startswith("NVML")


def test_fixed_point_energy_unit_and_conversion():
    import torch
    from blond_b200.engine import Q32_MAX, default_energy_unit, to_fixed
    dE = torch.tensor([-3e7, 1e6, 2.5e7, 0.0], dtype=torch.float64)
    u = default_energy_unit(dE)
    assert u == pytest.approx(1.5 * 3e7 / Q32_MAX)
    q = to_fixed(dE, u)
    assert q.dtype == torch.int32
    assert int(q.abs().max()) <= Q32_MAX
    assert float((q.double() * u - dE).abs().max()) <= u / 2 * (1 + 1e-12)
    with pytest.raises(ValueError):
        to_fixed(dE, u / 2)  # 3e7 eV is then 3e9 counts
    assert default_energy_unit(torch.zeros(3, dtype=torch.float64)) > 0


def test_fixed_point_restatement_approaches_the_fp64_oracle():
    """The fixed-point oracle with a fine unit follows the FP64 oracle: after
    30 turns the energies agree to the rounding the grid adds (at most half
    a unit per turn), the times to that rounding carried by the drift
    (~1.6e-18 s per eV per turn: ~1e-17 s, 3e-9 of max|dt|), and the
    profiles to a particle or two."""
    import cpu_oracle as o
    from blond_b200.beam.beam import Proton
    from blond_b200.beam.distributions import _get_dE_from_dt, bigaussian_arrays
    from blond_b200.input_parameters.rf_parameters import RFStation
    from blond_b200.input_parameters.ring import Ring
    turns, n, S = 30, 20000, 256
    ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), turns)
    rf = RFStation(ring, [4620], [4.5e6], [0.0])
    centre = (rf.phi_s[0] - rf.phi_rf[0, 0]) / rf.omega_rf[0, 0]
    dt0, dE0 = bigaussian_arrays(n, 0.4e-9, _get_dE_from_dt(ring, rf, 0.4e-9), centre, 4)
    cuts = (centre - 1.25e-9, centre + 1.25e-9)
    edges = np.linspace(*cuts, S + 1)
    bc = (edges[:-1] + edges[1:]) / 2
    unit = 0.1  # eV: a grid of +-215 MeV
    q0 = np.rint(dE0 / unit).astype(np.int64)
    fdt, fq, fprof = o.track_oracle_fixed(dt0, q0, unit, ring, rf, cuts, bc, S, turns)
    odt, odE, oprof, _ = o.track_oracle(dt0, q0 * unit, ring, rf, cuts, bc, S, turns)
    assert np.max(np.abs(fq * unit - odE)) <= turns * unit
    assert np.max(np.abs(fdt - odt)) / np.max(np.abs(odt)) < 1e-8
    assert np.abs(fprof[-1] - oprof[-1]).sum() <= 2
