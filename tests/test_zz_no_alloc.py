"""blond_turn_f64_noalloc: one fused turn that allocates no device memory.

The entry point serves callers that must not call cudaMalloc -- a tracking
step embedded in a host application that owns the device's memory (an
online model, a framework with its own pooling allocator), where an
allocation could stall every stream on the device and would bypass the
host's memory accounting.  Its temporaries live in a fixed file-scope
device array (profiles up to 16384 slices).

The test calls it through the C ABI for two turns in a row and compares
each turn with the engine's ordinary path (blond_engine_run, which uses
memory the engine allocated) on the same input, and with the CPU oracle:
coordinates within 1e-12 normwise (the two device paths run the same
kernels, so they agree to the bit in practice), slice counts exact,
induced voltage within 1e-10 normwise.  Free device memory is the same
before and after every call after the first (the first call may load the
library's device code, which commits the fixed array).  The file name
makes pytest collect it last.
"""
import ctypes as ct

import numpy as np
import pytest
import torch
from scipy.constants import e as E_CHARGE

from conftest import normwise
from blond_b200 import _lib
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

N, S, TURNS = 100003, 1024, 2


def _p(t):
    return ct.c_void_p(t.data_ptr())


def _columns(rf, t):
    """Turn t's RF column (voltage, omega_rf, phi_rf) as device arrays."""
    return [torch.as_tensor(np.ascontiguousarray(getattr(rf, k)[:, t]), device="cuda")
            for k in ("voltage", "omega_rf", "phi_rf")]


def _turn_noalloc(lib, rf, dt, dE, t, cols, cuts, Z, n_fft, scale, prof_out, v_out):
    """One call of the entry point for turn t (RF column t, drift t+1)."""
    d = t + 1
    rc = lib.blond_turn_f64_noalloc(
        _p(dt), _p(dE), dt.numel(), rf.n_rf, float(rf.particle.charge),
        _p(cols[0]), _p(cols[1]), _p(cols[2]), float(-rf.delta_E[t]), 0,
        float(rf.t_rev[d]), float(rf.length_ratio), float(rf.alpha_order),
        float(rf.eta_0[d]), float(rf.eta_1[d]), float(rf.eta_2[d]),
        float(rf.alpha_0[d]), float(rf.alpha_1[d]), float(rf.alpha_2[d]),
        float(rf.beta[d]), float(rf.energy[d]), float(cuts[0]), float(cuts[1]), S,
        _p(Z), int(n_fft), float(scale), _p(prof_out), _p(v_out),
        ct.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert rc == 0, lib.blond_b200_last_error().decode()


@pytest.mark.parametrize("window", [(-1.25e-9, 1.25e-9), (-0.9e-9, 1.6e-9)])
def test_noalloc_turn_matches_engine_twice(cuda, window):
    import cpu_oracle as o
    lib = _lib.load()
    ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), TURNS + 1)
    rf = RFStation(ring, [4620], [4.5e6], [0.0])
    centre = (rf.phi_s[0] - rf.phi_rf[0, 0]) / rf.omega_rf[0, 0]
    dt0, dE0 = bigaussian_arrays(N, 0.4e-9, _get_dE_from_dt(ring, rf, 0.4e-9), centre, 3)
    intensity = 1e10
    cuts = (centre + window[0], centre + window[1])

    # the engine's ordinary path (memory allocated by blond_engine_create)
    beam = Beam(ring, N, intensity, dt=dt0, dE=dE0)
    prof = Profile(beam, CutOptions(cut_left=cuts[0], cut_right=cuts[1], n_slices=S))
    iv = InducedVoltageFreq(beam, prof, [Resonators(5e6, 1e9, 1.0)])
    tiv = TotalInducedVoltage(beam, prof, [iv])
    fused = FusedTracker(RingAndRFTracker(rf, beam), prof, tiv, precision="f64",
                         turns_per_graph=1)

    # the entry point without allocation, on its own copy of the bunch; every
    # device buffer the calls use exists before the first call
    dt = torch.from_numpy(dt0).cuda()
    dE = torch.from_numpy(dE0).cuda()
    prof_out = torch.zeros(S, dtype=torch.float64, device="cuda")
    v_out = torch.zeros(S, dtype=torch.float64, device="cuda")
    Z = iv.total_impedance.contiguous()
    scale = rf.particle.charge * E_CHARGE * beam.ratio
    cols = [_columns(rf, t) for t in range(TURNS + 1)]
    Zh = iv.total_impedance.cpu().numpy()

    for t in range(TURNS):  # two calls in a row
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        _turn_noalloc(lib, rf, dt, dE, t, cols[t], cuts, Z, iv.n_fft, scale, prof_out, v_out)
        if t > 0:
            assert torch.cuda.mem_get_info()[0] == free_before, "the call allocated memory"
        fused.track(1)
        fused.check()
        assert normwise(dt.cpu().numpy(), beam.dt.cpu().numpy()) < 1e-12
        assert normwise(dE.cpu().numpy(), beam.dE.cpu().numpy()) < 1e-12
        np.testing.assert_array_equal(prof_out.cpu().numpy(),
                                      fused.profile_tensor().cpu().numpy())
        assert normwise(v_out.cpu().numpy(),
                        fused.induced_voltage_tensor().cpu().numpy()) < 1e-10
        # the oracle: the same t + 1 turns on the CPU
        odt, odE, oprof, ov = o.track_oracle(
            dt0, dE0, ring, rf, cuts, prof.bin_centers, S, t + 1,
            impedance=(iv.n_fft, Zh), intensity=intensity)
        assert normwise(dt.cpu().numpy(), odt) < 1e-12
        assert normwise(dE.cpu().numpy(), odE) < 1e-12
        np.testing.assert_array_equal(prof_out.cpu().numpy(), oprof[-1])
        assert normwise(v_out.cpu().numpy(), ov[-1]) < 1e-10

    # a later call, after the engine's own launches, allocates nothing either
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    _turn_noalloc(lib, rf, dt, dE, TURNS, cols[TURNS], cuts, Z, iv.n_fft, scale, prof_out,
                  v_out)
    assert torch.cuda.mem_get_info()[0] == free_before, "the call allocated memory"


def test_noalloc_rejects_profiles_beyond_its_scratch(cuda):
    lib = _lib.load()
    big = 16385
    dt = torch.zeros(16, dtype=torch.float64, device="cuda")
    v = torch.zeros(4, dtype=torch.float64, device="cuda")
    out = torch.zeros(big, dtype=torch.float64, device="cuda")
    rc = lib.blond_turn_f64_noalloc(
        _p(dt), _p(dt.clone()), 16, 1, 1.0, _p(v), _p(v), _p(v), 0.0, 0,
        *([1.0] * 11), 0.0, 1e-9, big, None, 0, 0.0, _p(out), None, None)
    assert rc == 2  # BLOND_ERR_SIZE
    assert "16384" in lib.blond_b200_last_error().decode()
