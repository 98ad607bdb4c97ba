"""The reference's own GPU kernels (blond/gpu/kernels.cu rebuilt for
sm_100a, oracle/ref_gpu.py) against the fused engine on the same inputs.

The reference build uses --use_fast_math, which lets nvcc contract its
FP64 drift and kick into FMAs; the engine evaluates the CPU reference's
expressions without contraction.  Bars: dt/dE within 1e-11 normwise after
10 turns of the full pipeline (induced voltage, interpolated kick, RF kick,
drift, slicing), profiles within a few particles (a contracted drift can
move a particle across a bin edge).  Skipped when the reference kernels
were not built (no reference checkout when oracle/ was made).
"""
import numpy as np
import pytest
import torch

import ref_cpu
import ref_gpu
from conftest import normwise
from blond_b200.beam.beam import Beam, Proton
from blond_b200.beam.distributions import _get_dE_from_dt, bigaussian_arrays
from blond_b200.beam.profile import CutOptions, Profile
from blond_b200.engine import FusedTracker
from blond_b200.impedances.impedance import InducedVoltageFreq, TotalInducedVoltage
from blond_b200.impedances.impedance_sources import Resonators
from blond_b200.input_parameters.rf_parameters import RFStation
from blond_b200.input_parameters.ring import Ring
from blond_b200.trackers.tracker import RingAndRFTracker

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_gpu.available(), reason="reference GPU kernels not built")]


@pytest.mark.parametrize("S", [1024, 16384])
def test_reference_gpu_kernels_match_fused_engine(cuda, S):
    n, turns = 200_000, 10
    ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), turns)
    rf = RFStation(ring, [4620], [4.5e6], [0.0])
    centre = (rf.phi_s[0] - rf.phi_rf[0, 0]) / rf.omega_rf[0, 0]
    dt0, dE0 = bigaussian_arrays(n, 0.4e-9, _get_dE_from_dt(ring, rf, 0.4e-9), centre, 2)
    beam = Beam(ring, n, 1e10, dt=dt0, dE=dE0)
    prof = Profile(beam, CutOptions(cut_left=centre - 1.25e-9, cut_right=centre + 1.25e-9,
                                    n_slices=S))
    iv = InducedVoltageFreq(beam, prof, [Resonators(5e6, 1e9, 1.0)])
    tiv = TotalInducedVoltage(beam, prof, [iv])
    ref = ref_gpu.RefGpuPath()
    ref.setup(ref_cpu.programme(rf), turns)
    rdt = torch.tensor(dt0, device="cuda")
    rdE = torch.tensor(dE0, device="cuda")
    rprof = torch.zeros(S, dtype=torch.float64, device="cuda")
    cuts = (float(prof.cut_left), float(prof.cut_right))
    bc = torch.tensor(np.asarray(prof.bin_centers), device="cuda")
    Z = iv.total_impedance.to("cuda")
    factor = torch.empty(2 * (S - 1), dtype=torch.float64, device="cuda")
    ref.slice(rdt, rprof, *cuts)
    for t in range(turns):
        ref.turn(t, rdt, rdE, rprof, cuts, bc, Z, iv.n_fft, 1.0, 1e10 / n, factor)
    fused = FusedTracker(RingAndRFTracker(rf, beam), prof, tiv, precision="f64")
    fused.track(turns)
    torch.cuda.synchronize()
    assert normwise(beam.dt.cpu().numpy(), rdt.cpu().numpy()) < 1e-11
    assert normwise(beam.dE.cpu().numpy(), rdE.cpu().numpy()) < 1e-11
    got, want = fused.profile_tensor().cpu().numpy(), rprof.cpu().numpy()
    assert got.sum() == want.sum() and np.abs(got - want).sum() <= 4
