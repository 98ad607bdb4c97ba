"""CPU BASELINE DRIVER -- test/benchmark infrastructure, not product code.

Times the reference's own CPU implementation of the per-turn path on the
host cores: the reference C++ kernels compiled from its sources into
oracle/_ref/libblond_ref_double.so (OpenMP, the `blond-compile --parallel
--optimize` flag set), driven in the call sequence of the reference objects
(TotalInducedVoltage.track -> RingAndRFTracker.track -> Profile.track, with
numpy.fft for the induced voltage exactly as bmath_backends.py:447-449
maps it).  Falls back to the plain-C restatement (oracle/_build/
liboracle.so, single-threaded) when the reference library was not built;
``kind`` reports which ran.
"""
from __future__ import annotations

import ctypes as ct
import os
import time

import numpy as np
from scipy.constants import e as E_CHARGE

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libblond_ref_double.so")
PORT_LIB = os.path.join(HERE, "_build", "liboracle.so")


class CpuPath:
    def __init__(self):
        if os.path.exists(REF_LIB):
            self.lib = ct.CDLL(REF_LIB)
            self.kind = "reference"
            self.names = dict(kick="kick", drift="drift", hist="histogram",
                              lik="linear_interp_kick")
            self.cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
        else:
            self.lib = ct.CDLL(PORT_LIB)
            self.kind = "port"
            self.names = dict(kick="oracle_kick_f64", drift="oracle_drift_f64",
                              hist="oracle_histogram_f64",
                              lik="oracle_linear_interp_kick_f64")
            self.cores = 1
        self.f = {k: getattr(self.lib, v) for k, v in self.names.items()}

    @staticmethod
    def _p(a):
        return a.ctypes.data_as(ct.c_void_p)

    def run(self, dt, dE, prog, n_turns, start_turn=0, impedance=None,
            cuts=None, bin_centers=None, n_slices=None, charge=1.0, ratio=1.0):
        """Track n_turns in place; returns seconds of wall time."""
        d = ct.c_double
        p = self._p
        n = len(dt)
        cl, cr = cuts
        prof = np.zeros(n_slices)
        bc = np.ascontiguousarray(bin_centers, dtype=np.float64)
        self.f["hist"](p(dt), p(prof), d(cl), d(cr), ct.c_int(n_slices), ct.c_int(n))
        t0 = time.perf_counter()
        for k in range(n_turns):
            t = start_turn + k
            if impedance is not None:
                n_fft, Z = impedance
                v = -(charge * E_CHARGE * ratio * np.fft.irfft(Z * np.fft.rfft(prof, n_fft)))
                v = np.ascontiguousarray(v[:n_slices])
                self.f["lik"](p(dt), p(dE), p(v), p(bc), d(charge), ct.c_int(n_slices),
                              ct.c_int(n), d(0.0))
            V, om, ph = (np.ascontiguousarray(prog[x][:, t]) for x in ("V", "om", "ph"))
            self.f["kick"](p(dt), p(dE), ct.c_int(len(V)), d(charge), p(V), p(om), p(ph),
                           ct.c_int(n), d(prog["acc"][t]))
            a = prog["drift"][t + 1]
            self.f["drift"](p(dt), p(dE), ct.c_int(0), *[d(x) for x in a], ct.c_int(n))
            self.f["hist"](p(dt), p(prof), d(cl), d(cr), ct.c_int(n_slices), ct.c_int(n))
        return time.perf_counter() - t0


def programme(rf):
    """Per-turn arrays the driver needs, from an RFStation-like object."""
    nt = rf.n_turns
    drift = [(rf.t_rev[t], rf.length_ratio, rf.alpha_order, rf.eta_0[t], rf.eta_1[t],
              rf.eta_2[t], rf.alpha_0[t], rf.alpha_1[t], rf.alpha_2[t], rf.beta[t],
              rf.energy[t]) for t in range(nt + 1)]
    return dict(V=np.asarray(rf.voltage, float), om=np.asarray(rf.omega_rf, float),
                ph=np.asarray(rf.phi_rf, float), acc=-np.asarray(rf.delta_E, float),
                drift=drift)
