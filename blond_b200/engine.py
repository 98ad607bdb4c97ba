"""Fused turn loop: the reference main loop in two launches per turn.

``FusedTracker`` takes the drop-in objects of one beam -- a
``RingAndRFTracker``, its ``Profile`` and optionally a
``TotalInducedVoltage`` -- and replaces

    for turn in range(n):                 # EX_05_Wake_impedance.py:336-339
        total_induced_voltage.track()     # impedance.py:133-146
        tracker.track()                   # tracker.py:521-615
        profile.track()                   # profile.py:700-719

by ``FusedTracker(...).track(n)``: per turn one cluster launch (profile ->
induced voltage -> interpolation table) and one pass over the particles
(induced kick, RF kick, drift, deposit), replayed from a CUDA graph.

Precision modes
---------------
'f64'    : dt, dE float64, everything float64 (the reference's arithmetic).
'f32p64' : dt float64, dE float32; the RF phase argument omega*dt+phi and
           the drift accumulate in float64, the kick in float32.  The
           engine keeps its own float32 energy array (``dE``).
'q32p64' : dt float64, dE int32 counts of an energy unit ``energy_unit``
           (eV); the kick and drift run in float64 and each turn's energy
           change is rounded once to the unit.  The default unit spans
           1.5 max|dE| of the initial bunch with the 2^31 - 1 counts of the
           grid (~0.1 eV for a 25 MeV rms bunch, 20 times finer than float32
           there); a particle that leaves the grid is reported by check().
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import torch
from scipy.constants import e

from . import _lib
from .impedances.impedance import (InducedVoltageFreq, InducedVoltageTime,
                                   InductiveImpedance)

PREC = {"f64": 0, "f32p64": 1, "q32p64": 2}

# counts on each side of 0 of the Q32P64 energy grid
Q32_MAX = 2**31 - 1


def default_energy_unit(dE) -> float:
    """Q32P64 energy unit for a bunch: 1.5 max|dE| over the grid's 2^31 - 1
    counts (1 keV of range at least)."""
    m = float(torch.as_tensor(dE).abs().max()) if torch.as_tensor(dE).numel() else 0.0
    return 1.5 * max(m, 1e3) / Q32_MAX


def to_fixed(dE: torch.Tensor, unit: float) -> torch.Tensor:
    """Energies (eV) as int32 counts of `unit` (round to nearest)."""
    q = torch.round(dE.to(torch.float64) / unit)
    if q.numel() and float(q.abs().max()) > Q32_MAX:
        raise ValueError("energies beyond the fixed-point grid; use a larger energy unit")
    return q.to(torch.int32).contiguous()
SOLVER = {"simple": 0, "legacy": 1, "exact": 2}


def _host(a) -> np.ndarray:
    if isinstance(a, torch.Tensor):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def _p(a: np.ndarray) -> ct.c_void_p:
    return a.ctypes.data_as(ct.c_void_p)


class TurnEngine:
    """Thin owner of a blond_engine handle (include/blond_b200.h)."""

    def __init__(self, precision: str, n_rf: int, solver: str, n_slices: int):
        _lib.load()
        self.h = ct.c_void_p()
        _lib.call("blond_engine_create", ct.byref(self.h), PREC[precision],
                  int(n_rf), SOLVER[solver], int(n_slices))
        self.n_slices = int(n_slices)
        self._keep = []

    def __del__(self):
        h = getattr(self, "h", None)
        if h is not None and h.value:
            try:
                _lib.load().blond_engine_destroy(h)
            except Exception:
                pass
            self.h = None

    def call(self, name, *args):
        _lib.call(f"blond_engine_{name}", self.h, *args)


# BeamFeedback.machine -> blond_engine_set_feedback code (include/blond_b200.h)
FB_MACHINES = {"LHC": 1, "LHC_F": 2, "SPS_F": 3, "SPS_RL": 4, "PSB": 5}


def _stream():
    return ct.c_void_p(torch.cuda.current_stream().cuda_stream)


def start_sharded(slice_local, reduce, refresh):
    """Initial profile of a beam split over ranks: slice the local
    particles, sum the histogram over the ranks, convert it."""
    slice_local()
    reduce()
    refresh()


def run_sharded_turns(n_turns, head, particles, reduce, refresh):
    """The turn loop of one beam split over ranks (the reference's MPI
    layout: Beam.split, beam/beam.py:626-697, and the per-turn histogram
    all-reduce of Profile.reduce_histo, beam/profile.py:721-762).

    Per turn, in this order on every rank (so every rank issues the same
    collectives): head() -- profile from the summed histogram, induced
    voltage, interpolation table; particles() -- the local particles'
    induced kick, RF kick, drift and deposit; reduce() -- sum the histogram
    over the ranks.  refresh() converts the final summed histogram."""
    for _ in range(int(n_turns)):
        head()
        particles()
        reduce()
    refresh()


class FusedTracker:
    def __init__(self, tracker, profile, total_induced_voltage=None,
                 precision: str = "f64", turns_per_graph: int = 50,
                 threads: int = 0, blocks_per_sm: int = 0, kernel: str = "auto",
                 process_group=None, tune: str | None = None,
                 energy_unit: float | None = None):
        if precision not in PREC:
            raise ValueError(f"precision must be one of {list(PREC)}")
        if tracker.interpolation and getattr(tracker, "profile", profile) is not profile:
            raise ValueError("an interpolated tracker interpolates over its own profile: "
                             "pass that profile")
        if getattr(profile, "smooth", False) and process_group is not None:
            raise NotImplementedError("smooth slicing of a sharded beam")
        rf = tracker.rf_params
        beam = tracker.beam
        self.tracker, self.profile, self.tiv = tracker, profile, total_induced_voltage
        self.rf, self.beam = rf, beam
        self.precision = precision
        S = int(profile.n_slices)
        self.eng = TurnEngine(precision, rf.n_rf, tracker.solver, S)
        nt = int(rf.n_turns)
        # programmes, turn-major (column t of the F-ordered [n_rf, n_turns+1])
        V = np.ascontiguousarray(np.asarray(rf.voltage, float).T)
        om = np.ascontiguousarray(np.asarray(rf.omega_rf, float).T)
        ph = np.ascontiguousarray(np.asarray(rf.phi_rf, float).T)
        acc = np.ascontiguousarray(np.asarray(tracker.acceleration_kick, float))
        self.eng.call("set_rf", nt, _p(V), _p(om), _p(ph), _p(acc),
                      float(rf.particle.charge))
        arr = [np.ascontiguousarray(np.asarray(getattr(rf, k), float))
               for k in ("t_rev", "eta_0", "eta_1", "eta_2", "alpha_0",
                         "alpha_1", "alpha_2", "beta", "energy")]
        self.eng.call("set_drift", float(rf.length_ratio), float(rf.alpha_order),
                      *[_p(a) for a in arr])
        bc = np.ascontiguousarray(np.asarray(profile.bin_centers, float))
        self.eng.call("set_slicing", float(profile.cut_left),
                      float(profile.cut_right), _p(bc))
        if total_induced_voltage is not None:
            self._set_impedance(total_induced_voltage, beam, rf)
        if tracker.interpolation:
            # RF + induced voltage interpolated from one table, no RF kick
            self.eng.call("set_interpolation", 1)
        if getattr(profile, "smooth", False):
            # slice_smooth weights, deposited after each particle pass
            self.eng.call("set_smooth", 1)
        self.loop = getattr(tracker, "beamFB", None)
        # coordinates
        if beam.dt.dtype != torch.float64:
            raise TypeError("the fused engine needs float64 dt")
        self.dt = beam.dt
        self.energy_unit = None
        if precision == "f64":
            if beam.dE.dtype != torch.float64:
                raise TypeError("precision 'f64' needs float64 dE")
            self.dE = beam.dE
        elif precision == "f32p64":
            self.dE = beam.dE.to(torch.float32).contiguous()
        else:
            if self.loop is not None and self.loop.machine == "SPS_RL":
                raise NotImplementedError("the SPS_RL loop with fixed-point energies")
            unit = float(energy_unit) if energy_unit else default_energy_unit(beam.dE)
            self.energy_unit = unit
            self.dE = to_fixed(beam.dE, unit)
            self.eng.call("set_energy_unit", unit)
        self.eng.call("bind_beam", ct.c_void_p(self.dt.data_ptr()),
                      ct.c_void_p(self.dE.data_ptr()), int(beam.n_macroparticles))
        self.eng.call("tune", int(threads), int(blocks_per_sm), int(turns_per_graph))
        if kernel not in ("auto", "tma", "plain", "stab", "packed"):
            raise ValueError("kernel must be 'auto', 'tma', 'plain', 'stab' (the plain "
                             "pass with the table in shared memory) or 'packed' (the plain "
                             "pass with a packed 16-bit histogram)")
        self.kernel_requested = kernel
        if kernel == "auto":
            # measured on the B200 (C2 workload): plain loads win for FP64
            # (87 vs 107 us), the bulk-copy pipeline ties or wins for F32P64
            kernel = "plain" if precision == "f64" else "tma"
        self.kernel = kernel
        self.eng.call("set_kernel", {"tma": 0, "plain": 1, "stab": 2, "packed": 3}[kernel])
        # the autotuner picks block size, grid (particles per thread),
        # histogram layout and staged vs plain pass on the first track() or
        # prepare(), unless the caller fixed any of them
        if tune is None:
            tune = "auto" if (self.kernel_requested == "auto" and not threads
                              and not blocks_per_sm) else "fixed"
        if tune not in ("auto", "fixed"):
            raise ValueError("tune must be 'auto' or 'fixed'")
        self.tune_mode = tune
        self.tuned = None
        self.eng.call("set_turn", int(rf.counter[0]), _stream())
        if self.loop is not None:
            self._set_loop(self.loop, process_group)
        # sharded: this rank holds a part of the beam; the int32 histogram is
        # summed over `process_group` after every particle pass.  The beam's
        # ratio (intensity / macro-particles) must be the whole beam's.
        self.group = process_group
        if process_group is None:
            self.eng.call("slice", _stream())
        else:
            self.hist = torch.zeros(S, dtype=torch.int32, device="cuda")
            self.eng.call("bind_histogram", ct.c_void_p(self.hist.data_ptr()))
            start_sharded(lambda: self.eng.call("slice", _stream()), self._reduce,
                          lambda: self.eng.call("step", 3, _stream()))

    def _set_loop(self, loop, process_group):
        """The beam-phase loop on the device (blond_engine_set_feedback):
        its per-turn table, parameters and current state from the
        BeamFeedback object (blond_b200.llrf.beam_feedback)."""
        if loop.RFnoise is not None or loop.noiseFB is not None:
            raise NotImplementedError("phase noise in the fused beam-phase loop")
        if loop.machine == "SPS_RL" and process_group is not None:
            raise NotImplementedError("the SPS_RL loop averages dE over the whole beam; "
                                      "not on a sharded beam")
        if loop.machine == "SPS_RL" and loop.reference != 0:
            raise NotImplementedError("radial steering (reference != 0)")
        code = FB_MACHINES[loop.machine]
        rf, ring = self.rf, loop.ring
        nt1 = int(rf.n_turns) + 1
        n_rf = rf.n_rf

        def col(x):
            return np.broadcast_to(np.asarray(x, dtype=float), (nt1,))
        zeros = np.zeros(nt1)
        gain = col(loop.gain)
        g2 = loop.gain2
        g2a, g2b = (col(g2[0]), col(g2[1])) if loop.machine == "PSB" else (zeros, zeros)
        lhc_a = col(loop.lhc_a) if loop.machine == "LHC" else zeros
        lhc_t = col(loop.lhc_t) if loop.machine == "LHC" else zeros
        table = np.column_stack(
            [col(rf.phi_s), col(rf.eta_0), col(np.asarray(ring.alpha_0)[0]), col(rf.gamma),
             col(np.asarray(ring.beta)[0]), col(np.asarray(ring.energy)[0]), lhc_a, lhc_t,
             gain, g2a, g2b]
            + [np.asarray(rf.omega_rf_d, float)[j, :nt1] for j in range(n_rf)]
            + [np.asarray(rf.harmonic, float)[j, :nt1] for j in range(n_rf)])
        table = np.ascontiguousarray(table, dtype=np.float64)
        state = np.zeros(16 + n_rf)
        if loop.machine == "LHC":
            state[0] = loop.lhc_y
        if loop.machine == "PSB":
            state[1:8] = (loop.dphi_sum, loop.dphi_av, loop.dphi_av_prev, loop.domega_PL,
                          loop.domega_RL, loop.dR_over_R_prev, loop.PL_counter)
            state[12] = loop.dR_over_R
        state[8:12] = (loop.phi_beam, loop.dphi, loop.domega_rf, loop.drho)
        state[16:] = np.asarray(rf.dphi_rf, float)
        on_time = np.ascontiguousarray(getattr(loop, "on_time", np.zeros(1)), dtype=np.float64)
        if on_time.size == 0:
            on_time = np.zeros(1)
        gain2 = 0.0 if loop.machine == "PSB" else float(loop.gain2)
        gain1 = 0.0 if loop.machine == "PSB" else float(loop.gain)
        self.eng.call("set_feedback", code, int(loop.delay), gain1, gain2,
                      float(loop.alpha), 1 if loop.time_offset is not None else 0,
                      float(loop.time_offset or 0.0), float(self.profile.bin_size),
                      float(ring.ring_radius), int(getattr(loop, "sample_dE", 1)),
                      _p(table), _p(on_time), int(on_time.size), _p(state))
        self._fb_n_state = state.size

    def _pull_loop(self):
        """The device loop's state and the corrected RF programmes back into
        the BeamFeedback and RFStation objects (what the host loop leaves);
        part of sync()."""
        if self.loop is None:
            return
        rf, loop = self.rf, self.loop
        nt1, n_rf = int(rf.n_turns) + 1, rf.n_rf
        st = torch.empty(self._fb_n_state, dtype=torch.float64, device="cuda")
        om = torch.empty((nt1, n_rf), dtype=torch.float64, device="cuda")
        ph = torch.empty_like(om)
        tr = torch.empty((nt1, 3), dtype=torch.float64, device="cuda")
        self.eng.call("get_feedback", ct.c_void_p(st.data_ptr()), ct.c_void_p(om.data_ptr()),
                      ct.c_void_p(ph.data_ptr()), ct.c_void_p(tr.data_ptr()), _stream())
        st, om, ph, tr = (x.cpu().numpy() for x in (st, om, ph, tr))
        rf.omega_rf[:, :] = om.T
        rf.phi_rf[:, :] = ph.T
        rf.dphi_rf[:] = st[16:16 + n_rf]
        loop.phi_beam, loop.dphi, loop.domega_rf = float(st[8]), float(st[9]), float(st[10])
        if loop.machine == "LHC":
            loop.lhc_y = float(st[0])
        elif loop.machine == "SPS_RL":
            loop.average_dE, loop.drho = float(st[13]), float(st[11])
        elif loop.machine == "PSB":
            (loop.dphi_sum, loop.dphi_av, loop.dphi_av_prev, loop.domega_PL, loop.domega_RL,
             loop.dR_over_R_prev) = (float(x) for x in st[1:7])
            loop.PL_counter = int(st[7])
            loop.dR_over_R = float(st[12])
        self.loop_trace = tr
        self.tracker._dev_prog = None  # the drop-in tracker re-sends the programmes

    def _reduce(self):
        import torch.distributed as dist
        dist.all_reduce(self.hist, op=dist.ReduceOp.SUM, group=self.group)

    def _set_impedance(self, tiv, beam, rf):
        Z = None
        n_fft = None
        for obj in tiv.induced_voltage_list:
            if isinstance(obj, InductiveImpedance):
                zn = np.ascontiguousarray(np.asarray(obj.Z_over_n, float))
                scale = beam.particle.charge * e / (2 * np.pi) * beam.ratio
                self._zn = zn
                self._ind_scale = scale
                continue
            if not isinstance(obj, (InducedVoltageFreq, InducedVoltageTime)):
                raise NotImplementedError(type(obj).__name__)
            if getattr(obj, "multi_turn_wake", False):
                raise NotImplementedError(
                    "multi-turn wakes: track with TotalInducedVoltage and "
                    "RingAndRFTracker instead of the fused engine")
            if n_fft is not None and obj.n_fft != n_fft:
                raise NotImplementedError("contributions with different n_fft")
            n_fft = obj.n_fft
            zi = _host(obj.total_impedance).astype(np.complex128)
            Z = zi if Z is None else Z + zi
        if Z is None:
            raise NotImplementedError("an inductive impedance alone needs an FFT "
                                      "impedance in the fused engine")
        if n_fft < self.profile.n_slices:
            raise NotImplementedError("n_fft shorter than the profile")
        self._Z = np.ascontiguousarray(Z)
        self.eng.call("set_impedance", int(n_fft), _p(self._Z.view(np.float64)),
                      float(beam.particle.charge * e * beam.ratio))
        if hasattr(self, "_zn"):
            self.eng.call("set_inductive", _p(self._zn), float(self._ind_scale))

    def autotune(self, reps: int = 3) -> dict:
        """Run the engine's autotuner now (blond_engine_autotune): times
        every feasible particle-pass configuration on this beam, keeps the
        fastest, then whole turns with and without the early launch of each
        turn's next kernel ('overlap'), and leaves the beam and the turn
        state untouched.  Returns the choice."""
        cfg = (ct.c_int * 9)()
        ms = ct.c_double()
        self.eng.call("autotune", int(reps), _stream(), cfg, ct.byref(ms))
        names = {-1: "auto", 0: "smem-warp-aggregated", 1: "smem-int", 2: "smem-packed16",
                 3: "global"}
        self.tuned = {"kernel": {0: "tma", 1: "plain", 2: "stab", 3: "packed"}[cfg[0]],
                      "threads": cfg[1],
                      "blocks_per_sm": cfg[2], "histogram": names.get(cfg[3], cfg[3]),
                      "prefetch_stages": cfg[4], "cluster": cfg[5],
                      "l2_prefetch": bool(cfg[6]), "candidates": cfg[7],
                      "overlap": bool(cfg[8]),
                      "particle_pass_ms": ms.value}
        self.kernel = self.tuned["kernel"]
        return self.tuned

    def _maybe_tune(self):
        if self.tune_mode == "auto" and self.tuned is None:
            self.autotune()

    def track(self, n_turns: int = 1):
        """Advance n_turns; updates the RF counter and beam energy fields."""
        self._maybe_tune()
        if self.group is None:
            self.eng.call("run", int(n_turns), _stream())
        else:
            run_sharded_turns(n_turns, lambda: self.eng.call("step", 1, _stream()),
                              lambda: self.eng.call("step", 2, _stream()), self._reduce,
                              lambda: self.eng.call("step", 3, _stream()))
        rf = self.rf
        rf.counter[0] += int(n_turns)
        t = rf.counter[0]
        self.beam.beta = float(rf.beta[t])
        self.beam.gamma = float(rf.gamma[t])
        self.beam.energy = float(rf.energy[t])
        self.beam.momentum = float(rf.momentum[t])

    def track_host(self, host_dt: torch.Tensor, host_dE: torch.Tensor, n_turns: int = 1,
                   chunks: int = 4):
        """Advance n_turns on coordinates held in (pinned) host tensors:
        every turn copies them in, tracks and copies them back, pipelined in
        chunks against the particle pass (blond_engine_track_host)."""
        edt = {"f64": torch.float64, "f32p64": torch.float32,
               "q32p64": torch.int32}[self.precision]
        if host_dt.device.type != "cpu" or host_dE.device.type != "cpu":
            raise ValueError("track_host takes host tensors")
        if host_dt.dtype != torch.float64 or host_dE.dtype != edt:
            raise TypeError(f"host arrays must be float64 dt and {edt} dE")
        if host_dt.numel() != self.dt.numel() or host_dE.numel() != self.dE.numel():
            raise ValueError("host arrays must hold the bound beam")
        if not (host_dt.is_contiguous() and host_dE.is_contiguous()):
            raise ValueError("host arrays must be contiguous")
        self._maybe_tune()
        self.eng.call("track_host", ct.c_void_p(host_dt.data_ptr()),
                      ct.c_void_p(host_dE.data_ptr()), int(n_turns), int(chunks), _stream())
        rf = self.rf
        rf.counter[0] += int(n_turns)
        t = rf.counter[0]
        self.beam.beta = float(rf.beta[t])
        self.beam.gamma = float(rf.gamma[t])
        self.beam.energy = float(rf.energy[t])
        self.beam.momentum = float(rf.momentum[t])

    def prepare(self):
        """Build and upload the CUDA graph now (otherwise the first track()
        of at least turns_per_graph turns builds it)."""
        self._maybe_tune()
        self.eng.call("prepare", _stream())

    def check(self):
        """Synchronise and raise if a kernel's bounded wait gave up."""
        self.eng.call("check", _stream())

    def time_kernels(self, n_turns: int):
        """Track n_turns with CUDA events around each launch; returns the
        summed (head_ms, particles_ms).  Synchronises the current stream."""
        self._maybe_tune()
        h, p = ct.c_double(), ct.c_double()
        self.eng.call("time_kernels", int(n_turns), ct.byref(h), ct.byref(p), _stream())
        self.rf.counter[0] += int(n_turns)
        return h.value, p.value

    def sync(self):
        """Copy the engine's profile (and induced voltage) into the drop-in
        objects, the float32 energies back into beam.dE ('f32p64'), and a
        beam-phase loop's state and corrected RF programmes into the
        BeamFeedback and RFStation objects."""
        self.check()
        prof = torch.empty(self.profile.n_slices, dtype=torch.float64, device="cuda")
        self.eng.call("get_profile", ct.c_void_p(prof.data_ptr()), _stream())
        self.profile.n_macroparticles.copy_(prof)
        if self.tiv is not None:
            v = torch.empty_like(prof)
            self.eng.call("get_induced_voltage", ct.c_void_p(v.data_ptr()), _stream())
            self.tiv.induced_voltage = v.to(self.profile.n_macroparticles.dtype)
        if self.precision != "f64":
            self.beam.dE.copy_(self.energies())
        self._pull_loop()

    def energies(self) -> torch.Tensor:
        """The engine's energies in eV as a float64 device tensor (for
        'q32p64' the counts times the energy unit)."""
        if self.precision == "q32p64":
            return self.dE.to(torch.float64) * self.energy_unit
        return self.dE.to(torch.float64)

    def profile_tensor(self) -> torch.Tensor:
        prof = torch.empty(self.profile.n_slices, dtype=torch.float64, device="cuda")
        self.eng.call("get_profile", ct.c_void_p(prof.data_ptr()), _stream())
        return prof

    def induced_voltage_tensor(self) -> torch.Tensor:
        v = torch.empty(self.profile.n_slices, dtype=torch.float64, device="cuda")
        self.eng.call("get_induced_voltage", ct.c_void_p(v.data_ptr()), _stream())
        return v
