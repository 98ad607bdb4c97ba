"""CPU checks of the beam-phase restatement (oracle/blond_oracle.c
oracle_beam_phase_*) against the reference's compiled beam_phase /
beam_phase_fast (cpp_routines/beam_phase.cpp:6-65), stored in
tests/golden/beam_phase.npz by tests/golden/gen_golden.py.

Bars: float64 1e-13 relative (the reference's OpenMP sum and VDT sine
against a serial sum and libm); float32 1e-4 relative (the two-bin case
divides nearly cancelling float sums)."""
import numpy as np
import pytest

import cpu_oracle as co
from conftest import golden


@pytest.mark.parametrize("tag", ["f64", "f32"])
def test_oracle_beam_phase_matches_reference(tag):
    g = golden("beam_phase.npz")
    rtol = 1e-13 if tag == "f64" else 1e-4
    for k, (want_w, want_f) in enumerate(g[f"{tag}_coeff"]):
        bc, p = g[f"{tag}_{k}_bc"], g[f"{tag}_{k}_profile"]
        alpha, om, ph, bs = g[f"{tag}_{k}_params"]
        got_w = co.beam_phase(bc, p, alpha, om, ph, bs, weighted=True)
        got_f = co.beam_phase(bc, p, 0.0, om, ph, bs, weighted=False)
        np.testing.assert_allclose(got_w, want_w, rtol=rtol)
        np.testing.assert_allclose(got_f, want_f, rtol=rtol)
