"""blond_b200 -- B200-native longitudinal tracking hot path for BLonD.

Drop-in counterparts of the reference's per-turn objects live under the
same module paths as in the reference package:

    blond_b200.input_parameters.ring.Ring
    blond_b200.input_parameters.rf_parameters.RFStation
    blond_b200.beam.beam.Beam / Proton
    blond_b200.beam.distributions.bigaussian
    blond_b200.beam.profile.Profile / CutOptions
    blond_b200.impedances.impedance.TotalInducedVoltage / InducedVoltageFreq /
        InducedVoltageTime / InductiveImpedance
    blond_b200.impedances.impedance_sources.Resonators
    blond_b200.trackers.tracker.RingAndRFTracker

``blond_b200.bmath`` holds the bmath-level kernels (kick, drift,
slice_beam, ...) and ``blond_b200.engine.FusedTracker`` the fused turn loop.
All compute runs in libblond_b200.so (sm_100a); there is no CPU fallback.
"""
from . import _lib  # noqa: F401
from ._lib import BlondB200Error  # noqa: F401

__version__ = "0.1.0"


def library_path() -> str:
    from .build import LIB
    return LIB
