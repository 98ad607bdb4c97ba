"""Many independent beams tracked together (one launch per turn for all).

In the reference every beam is its own set of objects -- a
RingAndRFTracker, a Profile and a TotalInducedVoltage -- tracked by its own
loop (__EXAMPLES/main_files/EX_05_Wake_impedance.py:318-339).  A parameter
scan over hundreds of such beams (different voltages, bunch lengths,
impedances; ragged particle counts) then costs hundreds of small launches
per turn.  ``BatchTracker`` takes the drop-in objects of all beams and
tracks them with the batched engine (blond_batch_*): one particle pass and
one head launch (one FFT cluster per beam) per turn, replayed from a CUDA
graph, each beam with the single-beam engine's arithmetic.

All beams must share the number of RF systems, the drift solver, the
number of slices, the programme length and (when present) the FFT length
of the impedance; everything else may differ per beam.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import torch
from scipy.constants import e

from . import _lib
from .engine import PREC, SOLVER, _host, default_energy_unit, to_fixed
from .impedances.impedance import InducedVoltageFreq, InducedVoltageTime


def _p(a: np.ndarray) -> ct.c_void_p:
    return a.ctypes.data_as(ct.c_void_p)


def _stream():
    return ct.c_void_p(torch.cuda.current_stream().cuda_stream)


class BatchTracker:
    def __init__(self, items, precision: str = "f32p64", turns_per_graph: int = 50,
                 energy_units=None):
        """items: list of (RingAndRFTracker, Profile, TotalInducedVoltage or
        None), one per beam.  'q32p64' stores each beam's energies as int32
        counts of its own unit (energy_units, eV; by default 1.5 max|dE| of
        the beam over the 2^31 - 1 counts of the grid)."""
        if precision not in PREC:
            raise ValueError(f"precision must be one of {list(PREC)}")
        self.items = list(items)
        if not self.items:
            raise ValueError("empty batch")
        trackers = [t for t, _, _ in self.items]
        profiles = [p for _, p, _ in self.items]
        tivs = [v for _, _, v in self.items]
        rfs = [t.rf_params for t in trackers]
        beams = [t.beam for t in trackers]
        B = len(self.items)
        n_rf, S, nt = rfs[0].n_rf, int(profiles[0].n_slices), int(rfs[0].n_turns)
        solver = trackers[0].solver
        for t, p, rf in zip(trackers, profiles, rfs):
            if t.interpolation:
                raise NotImplementedError("the batched engine tracks the non-interpolated kick")
            if getattr(t, "beamFB", None) is not None:
                raise NotImplementedError("a beam-phase loop: track with RingAndRFTracker")
            if rf.n_rf != n_rf or int(p.n_slices) != S or int(rf.n_turns) != nt \
                    or t.solver != solver:
                raise ValueError("beams of a batch must share n_rf, n_slices, n_turns "
                                 "and the drift solver")
            if rf.counter[0] != rfs[0].counter[0]:
                raise ValueError("beams of a batch must be at the same turn")
        if any(v is None for v in tivs) and not all(v is None for v in tivs):
            raise ValueError("either every beam or no beam has an induced voltage")
        self.B, self.S, self.precision = B, S, precision
        self.rfs, self.beams, self.profiles, self.tivs = rfs, beams, profiles, tivs
        _lib.load()
        self.h = ct.c_void_p()
        _lib.call("blond_batch_create", ct.byref(self.h), PREC[precision], B, n_rf,
                  SOLVER[solver], S)
        self._call("tune", int(turns_per_graph))
        # programmes, beam-major
        V = np.ascontiguousarray(np.stack([np.asarray(r.voltage, float).T for r in rfs]))
        om = np.ascontiguousarray(np.stack([np.asarray(r.omega_rf, float).T for r in rfs]))
        ph = np.ascontiguousarray(np.stack([np.asarray(r.phi_rf, float).T for r in rfs]))
        acc = np.ascontiguousarray(np.stack([-np.asarray(r.delta_E, float) for r in rfs]))
        self._call("set_rf", nt, _p(V), _p(om), _p(ph), _p(acc),
                   float(rfs[0].particle.charge))
        self._keep = [V, om, ph, acc]
        arr = [np.ascontiguousarray(np.stack([np.asarray(getattr(r, k), float)
                                              for r in rfs]))
               for k in ("t_rev", "eta_0", "eta_1", "eta_2", "alpha_0", "alpha_1",
                         "alpha_2", "beta", "energy")]
        self._call("set_drift", float(rfs[0].length_ratio), float(rfs[0].alpha_order),
                   *[_p(a) for a in arr])
        cl = np.array([p.cut_left for p in profiles], float)
        cr = np.array([p.cut_right for p in profiles], float)
        bc = np.ascontiguousarray(np.stack([np.asarray(p.bin_centers, float)
                                            for p in profiles]))
        self._call("set_slicing", _p(cl), _p(cr), _p(bc))
        if tivs[0] is not None:
            Z, n_fft = [], None
            for v in tivs:
                zb = None
                for obj in v.induced_voltage_list:
                    if not isinstance(obj, (InducedVoltageFreq, InducedVoltageTime)):
                        raise NotImplementedError(type(obj).__name__)
                    if n_fft is not None and obj.n_fft != n_fft:
                        raise ValueError("beams of a batch must share n_fft")
                    n_fft = obj.n_fft
                    zi = _host(obj.total_impedance).astype(np.complex128)
                    zb = zi if zb is None else zb + zi
                Z.append(zb)
            Z = np.ascontiguousarray(np.stack(Z))
            scale = np.array([b.particle.charge * e * b.ratio for b in beams], float)
            self._call("set_impedance", int(n_fft), _p(Z.view(np.float64)), _p(scale))
            self._keep += [Z, scale]
        # coordinates of all beams, concatenated on the device
        counts = [b.n_macroparticles for b in beams]
        self.offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        self.dt = torch.cat([b.dt.to(torch.float64) for b in beams]).contiguous()
        self.energy_units = None
        if precision == "q32p64":
            units = (list(energy_units) if energy_units is not None
                     else [default_energy_unit(b.dE) for b in beams])
            if len(units) != B:
                raise ValueError("one energy unit per beam")
            self.energy_units = np.ascontiguousarray(units, dtype=np.float64)
            self.dE = torch.cat([to_fixed(b.dE, u) for b, u in zip(beams, units)]).contiguous()
            self._call("set_energy_units", _p(self.energy_units))
        else:
            edtype = torch.float64 if precision == "f64" else torch.float32
            self.dE = torch.cat([b.dE.to(edtype) for b in beams]).contiguous()
        self._call("bind_beams", ct.c_void_p(self.dt.data_ptr()),
                   ct.c_void_p(self.dE.data_ptr()), _p(self.offsets))
        self.shape = None
        self._call("set_turn", int(rfs[0].counter[0]), _stream())
        self._call("slice", _stream())

    def _call(self, name, *args):
        _lib.call(f"blond_batch_{name}", self.h, *args)

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            try:
                _lib.load().blond_batch_destroy(h)
            except Exception:
                pass
            self.h = None

    def prepare(self):
        """Build and upload the CUDA graph now (else the first track() of at
        least turns_per_graph turns builds it)."""
        self._call("prepare", _stream())

    def set_shape(self, threads: int = 512, blocks_per_sm: int = 2,
                  particles_per_thread: int = 4, chunk: int = 32768,
                  aggregate: bool = False):
        """Fix the particle pass's launch shape (blond_batch_set_shape)."""
        self._call("set_shape", int(threads), int(blocks_per_sm), int(particles_per_thread),
                   int(chunk), 1 if aggregate else 0)

    def autotune(self, reps: int = 3) -> dict:
        """Time every launch shape of the particle pass on these beams and
        keep the fastest (blond_batch_autotune); the coordinates are left
        as they were.  Returns the choice."""
        cfg = (ct.c_int * 6)()
        ms = ct.c_double()
        self._call("autotune", int(reps), _stream(), cfg, ct.byref(ms))
        self.shape = {"threads": cfg[0], "blocks_per_sm": cfg[1],
                      "particles_per_thread": cfg[2], "chunk": cfg[3],
                      "aggregate": bool(cfg[4]), "candidates": cfg[5],
                      "particle_pass_ms": ms.value}
        return self.shape

    def check(self):
        """Synchronise and raise if a fixed-point energy left its grid."""
        self._call("check", _stream())

    def track(self, n_turns: int = 1):
        self._call("run", int(n_turns), _stream())
        for rf, beam in zip(self.rfs, self.beams):
            rf.counter[0] += int(n_turns)
            t = rf.counter[0]
            beam.beta, beam.gamma = float(rf.beta[t]), float(rf.gamma[t])
            beam.energy, beam.momentum = float(rf.energy[t]), float(rf.momentum[t])

    def profiles_tensor(self) -> torch.Tensor:
        out = torch.empty(self.B, self.S, dtype=torch.float64, device="cuda")
        self._call("get_profiles", ct.c_void_p(out.data_ptr()), _stream())
        return out

    def induced_voltages_tensor(self) -> torch.Tensor:
        out = torch.empty(self.B, self.S, dtype=torch.float64, device="cuda")
        self._call("get_induced_voltages", ct.c_void_p(out.data_ptr()), _stream())
        return out

    def coordinates(self, b: int):
        """(dt, dE) device views of beam b inside the batch arrays (dE in
        the engine's storage type)."""
        o0, o1 = int(self.offsets[b]), int(self.offsets[b + 1])
        return self.dt[o0:o1], self.dE[o0:o1]

    def energies(self, b: int) -> torch.Tensor:
        """Beam b's energies in eV as a float64 device tensor."""
        dE = self.coordinates(b)[1].to(torch.float64)
        if self.precision == "q32p64":
            dE = dE * float(self.energy_units[b])
        return dE

    def sync(self):
        """Copy coordinates, profiles and induced voltages back into the
        drop-in objects of every beam."""
        prof = self.profiles_tensor()
        vind = self.induced_voltages_tensor() if self.tivs[0] is not None else None
        for b, (beam, p, v) in enumerate(zip(self.beams, self.profiles, self.tivs)):
            beam.dt.copy_(self.coordinates(b)[0])
            beam.dE.copy_(self.energies(b))
            p.n_macroparticles.copy_(prof[b])
            if v is not None:
                v.induced_voltage = vind[b].to(p.n_macroparticles.dtype)
