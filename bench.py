#!/usr/bin/env python
"""Benchmark of the per-turn longitudinal tracking path.

Workload (one "step" = one turn over the whole beam): protons at 26 GeV/c,
C = 6911.5 m, gamma_t = 18, h = 4620, V = 4.5 MV, phi = 0; bi-Gaussian bunch
(sigma_dt 0.4 ns, sigma_dE matched, seed 0) of 1e7 macro-particles,
intensity 1e10; 2^14 slices over 2.5 ns around the bunch centre; induced
voltage of a broadband resonator (R_s 5 MOhm, f_r 1 GHz, Q 1) through
InducedVoltageFreq (n_fft = 16384), applied with linear_interp_kick; then
the RF kick, the drift and the slicing.  Synthetic data only.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Our arm times K fused turns (CUDA graph) on the device with CUDA events and
prints one JSON line; --impl reference times the reference's CPU C++ path
(oracle/_ref) on the host cores with the same workload and metric.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-turns/s on 1 B200, FP32-batched vs plain FP64 at <=1e-5 rel err"
UNIT = "particle-turns/s"
WORKLOAD = ("1e7 protons 26 GeV/c, h=4620 4.5 MV, 2^14 slices, broadband "
            "resonator 5 MOhm/1 GHz/Q=1 via FFT (n_fft 16384), lik + kick + "
            "drift + slice per turn")
BYTES_PER_PARTICLE = {"f64": 32, "f32p64": 24, "q32p64": 24}  # read + write of dt and dE
E2E_CHUNKS = 4


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--particles", type=float, default=1e7)
    ap.add_argument("--slices", type=int, default=16384)
    ap.add_argument("--precision", default="f64", choices=["f64", "f32p64", "q32p64"])
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-batched", action="store_true",
                    help="leave the C3 batch out of the default line")
    ap.add_argument("--batched-error-turns", type=int, default=1000,
                    help="turns after which the batched forms' rms errors are taken")
    ap.add_argument("--kernel", default="auto", choices=["auto", "tma", "plain", "stab", "packed"])
    ap.add_argument("--workload", default="c2", choices=["c2", "c3", "c4", "c5", "mtw"],
                    help="c2: the single-beam pipeline (default, the headline); "
                         "c3: 256-beam double-RF batch; c4: adjoint gradient; "
                         "c5: 1e8 particles, "
                         "2^16 slices, 4 resonators + inductive Z/n; "
                         "mtw: one turn of InducedVoltageResonator's multi-turn wake")
    ap.add_argument("--beams", type=int, default=256)
    ap.add_argument("--feedback", default="none",
                    choices=["none", "LHC", "LHC_F", "SPS_F", "SPS_RL", "PSB"],
                    help="c2 with a beam-phase loop of this machine type in every turn")
    ap.add_argument("--tune", default="auto", choices=["auto", "fixed"],
                    help="fixed: no autotuner; --threads/--blocks-per-sm/--prefetch "
                         "give the particle pass's launch shape (profiling runs)")
    ap.add_argument("--threads", type=int, default=1024)
    ap.add_argument("--blocks-per-sm", type=int, default=1)
    ap.add_argument("--prefetch", type=int, default=2, choices=[0, 2, 4])
    ap.add_argument("--c3-forms", default="q32p64,f32p64,f64",
                    help="c3: the precision forms to run (q32p64 gives the line's value; "
                         "f64 also runs the beams one by one and the FP64 controls)")
    ap.add_argument("--particles-per-thread", type=int, default=4, choices=[2, 4, 8],
                    help="c3 with --tune fixed: particles per thread of the batched pass")
    ap.add_argument("--chunk", type=int, default=16384,
                    help="c3 with --tune fixed: particles per chunk of the batched pass")
    ap.add_argument("--c5-forms", default="q32p64,f32p64,f64,control",
                    help="c5: the forms to run (comma list of q32p64, f32p64, f64, control); "
                         "q32p64 gives the line's value")
    return ap.parse_args()


# ----------------------------------------------------------------- machine
def machine(n_turns: int):
    from blond_b200.beam.beam import Proton
    from blond_b200.input_parameters.rf_parameters import RFStation
    from blond_b200.input_parameters.ring import Ring
    ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), n_turns)
    rf = RFStation(ring, [4620], [4.5e6], [0.0])
    return ring, rf


def host_bunch(ring, rf, n: int, seed: int = 0):
    from blond_b200.beam.distributions import _get_dE_from_dt, bigaussian_arrays
    sdE = _get_dE_from_dt(ring, rf, 0.4e-9)
    centre = (rf.phi_s[0] - rf.phi_rf[0, 0]) / rf.omega_rf[0, 0]
    dt, dE = bigaussian_arrays(n, 0.4e-9, sdE, centre, seed)
    return dt, dE, centre


def window(centre, S):
    cl, cr = centre - 1.25e-9, centre + 1.25e-9
    edges = np.linspace(cl, cr, S + 1)
    return cl, cr, (edges[:-1] + edges[1:]) / 2


# ----------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock and clock-event reasons during the timed region.  NVML is
    polled about every millisecond from a host thread (the timed region of
    the default run lasts ~20 ms); without NVML, nvidia-smi samples every
    200 ms instead."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, device_index: int):
        self.rows = []
        self.proc = None
        self.nvml = None
        self.halt = threading.Event()
        try:
            self._start_nvml(device_index)
            return
        except Exception:  # no NVML: fall back to nvidia-smi
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(device_index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _start_nvml(self, device_index):
        import pynvml as nv
        import torch
        nv.nvmlInit()
        try:  # the CUDA device's own GPU, whatever CUDA_VISIBLE_DEVICES says
            h = nv.nvmlDeviceGetHandleByUUID(
                "GPU-" + str(torch.cuda.get_device_properties(device_index).uuid))
        except Exception:
            h = nv.nvmlDeviceGetHandleByIndex(device_index)
        self.nvml, self.h = nv, h
        self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        self.bits = [nv.nvmlClocksEventReasonHwSlowdown,
                     nv.nvmlClocksEventReasonHwThermalSlowdown,
                     nv.nvmlClocksEventReasonSwThermalSlowdown,
                     nv.nvmlClocksEventReasonSwPowerCap]
        self._sample()  # fails here, not in the thread, if NVML cannot read
        self.t = threading.Thread(target=self._poll, daemon=True)
        self.t.start()

    def _sample(self):
        nv, h = self.nvml, self.h
        mhz = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        self.rows.append((mhz, [bool(r & b) for b in self.bits]))

    def _poll(self):
        while not self.halt.is_set():
            try:
                self._sample()
            except Exception:
                return
            time.sleep(0.001)

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.nvml is not None:
            self.halt.set()
            self.t.join(timeout=5)
            try:
                self._sample()  # the state at the end of the timed region
            except Exception:
                pass
            rows = self.rows
            reasons = sorted({self.NAMES[i] for _, f in rows for i in range(4) if f[i]})
            return {"sm_mhz": statistics.median(m for m, _ in rows),
                    "sm_max_mhz": self.max_mhz, "reasons": reasons,
                    "samples": len(rows), "source": "NVML, ~1 ms polling"}
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = [r for r in self.rows if len(r) >= 7]
        if not rows:
            return None
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        reasons = sorted({self.NAMES[i] for r in rows for i in range(4)
                          if r[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][1]) if rows[0][1].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(rows), "source": "nvidia-smi, 200 ms"}


# ----------------------------------------------------------------- CPU path
def cpu_reference(n: int, S: int, turns: int | None, seconds: float | None,
                  warmup: int = 0):
    """Reference C++ (oracle/_ref) on the host cores; returns
    (particle-turns/s, turns timed, kind, cores)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_cpu
    path = ref_cpu.CpuPath()
    total = (turns or 1000) + warmup + 2
    ring, rf = machine(total)
    dt, dE, centre = host_bunch(ring, rf, n)
    cl, cr, bc = window(centre, S)
    bin_size = (cr - cl) / S
    freq = np.fft.rfftfreq(S, bin_size)
    Z = _resonator_host(path, freq) / bin_size
    prog = ref_cpu.programme(rf)
    kw = dict(impedance=(S, Z), cuts=(cl, cr), bin_centers=bc, n_slices=S,
              charge=1.0, ratio=1e10 / n)
    if warmup:
        path.run(dt, dE, prog, warmup, 0, **kw)
    if turns is None:
        # bounded sample: turns until about `seconds` of CPU work
        one = path.run(dt, dE, prog, 1, warmup, **kw)
        turns = max(1, min(total - warmup - 2, int(seconds / max(one, 1e-6))))
        sec = path.run(dt, dE, prog, turns, warmup + 1, **kw)
    else:
        sec = path.run(dt, dE, prog, turns, warmup, **kw)
    return n * turns / sec, turns, path.kind, path.cores, sec


def _resonator_host(path, freq, R=(5e6,), Q=(1.0,), fr=(1e9,)):
    """Impedance on the host with the reference's own fast_resonator (or the
    restatement when the reference library is absent)."""
    import ctypes as ct
    f = np.ascontiguousarray(freq, dtype=np.float64)
    re, im = np.zeros(len(f)), np.zeros(len(f))
    R, Q, fr = (np.ascontiguousarray(x, dtype=np.float64) for x in (R, Q, fr))
    P = lambda a: a.ctypes.data_as(ct.c_void_p)  # noqa: E731
    fn = getattr(path.lib, "fast_resonator_real_imag", None) or \
        getattr(path.lib, "oracle_fast_resonator_f64")
    fn(P(re), P(im), P(f), P(R), P(Q), P(fr), ct.c_int(len(R)), ct.c_int(len(f)))
    return re + 1j * im


# ----------------------------------------------------------------- dist
def dist_init(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        if args.impl == "ours":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def dist_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


# ----------------------------------------------------------------- our arm
FEEDBACK_CONFIGS = {
    "LHC": {"machine": "LHC", "PL_gain": 1000.0},
    "LHC_F": {"machine": "LHC_F", "PL_gain": 1000.0, "FL_gain": 0.05},
    "SPS_F": {"machine": "SPS_F", "PL_gain": 1000.0, "FL_gain": 0.05},
    "SPS_RL": {"machine": "SPS_RL", "PL_gain": 1000.0, "RL_gain": 1e6, "sample_dE": 1},
    "PSB": {"machine": "PSB", "PL_gain": 1000.0, "RL_gain": [1e4, 1e2], "period": 1e-4},
}


def build_fused(n, S, n_turns, precision, kernel="auto", seed=0, group=None, shape=None,
                feedback="none"):
    """One beam of n macro-particles per GPU.  With a process group the GPUs
    hold shards of ONE beam (seed = rank: independent samples of the same
    bunch) whose histogram is summed every turn; the charge per
    macro-particle (1e10 / 1e7) is the same in every configuration."""
    import torch
    from blond_b200.beam.beam import Beam
    from blond_b200.beam.profile import CutOptions, Profile
    from blond_b200.engine import FusedTracker
    from blond_b200.impedances.impedance import InducedVoltageFreq, TotalInducedVoltage
    from blond_b200.impedances.impedance_sources import Resonators
    from blond_b200.trackers.tracker import RingAndRFTracker
    ring, rf = machine(n_turns)
    dt, dE, centre = host_bunch(ring, rf, n, seed)
    beam = Beam(ring, n, 1e10 * n / 1e7, dt=dt, dE=dE, dtype=torch.float64)
    cl, cr, _ = window(centre, S)
    prof = Profile(beam, CutOptions(cut_left=cl, cut_right=cr, n_slices=S))
    iv = InducedVoltageFreq(beam, prof, [Resonators(5e6, 1e9, 1.0)])
    tiv = TotalInducedVoltage(beam, prof, [iv])
    loop = None
    if feedback != "none":
        from blond_b200.llrf.beam_feedback import BeamFeedback
        cfg = {k: (list(v) if isinstance(v, list) else v)
               for k, v in FEEDBACK_CONFIGS[feedback].items()}
        loop = BeamFeedback(ring, rf, prof, cfg)
    tracker = RingAndRFTracker(rf, beam, beam_feedback=loop)
    if shape is None:
        fused = FusedTracker(tracker, prof, tiv, precision=precision, turns_per_graph=50,
                             kernel=kernel, process_group=group)
    else:
        threads, bps, ring = shape
        fused = FusedTracker(tracker, prof, tiv, precision=precision, turns_per_graph=50,
                             kernel="plain" if kernel == "auto" else kernel, threads=threads,
                             blocks_per_sm=bps, process_group=group, tune="fixed")
        fused.eng.call("set_prefetch", ring)
    return fused, beam, iv.n_fft


def time_turns(fused, turns):
    import torch
    s = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(s)
    fused.track(turns)
    b.record(s)
    torch.cuda.synchronize()
    return a.elapsed_time(b)


def run_ours(args, world, rank, local):
    import torch
    n = int(args.particles)
    S = args.slices
    W, K = max(3, args.warmup), args.steps
    kt = min(K, 20)
    E = args.e2e_steps
    total = W + K + kt + E + 5
    group = None
    if world > 1:
        import torch.distributed as dist
        group = dist.group.WORLD
    shape = ((args.threads, args.blocks_per_sm, args.prefetch) if args.tune == "fixed"
             else None)
    fused, beam, n_fft = build_fused(n, S, total, args.precision, args.kernel, seed=rank,
                                     group=group, shape=shape, feedback=args.feedback)
    fused.track(W)
    if group is None:
        fused.prepare()  # graph capture/upload outside the timed region
    torch.cuda.synchronize()
    barrier(world)
    clocks = ClockSampler(local) if rank == 0 else None
    ms = time_turns(fused, K)
    clk = clocks.stop() if clocks else None
    ms_max = dist_max(ms, world)
    value = world * n * K / (ms_max * 1e-3)
    # kernel durations (non-graph launches bracketed by events)
    fused.check()
    head_ms, part_ms = fused.time_kernels(kt)
    part_avg = part_ms / kt
    head_avg = head_ms / kt
    alg_bytes = BYTES_PER_PARTICLE[args.precision] * n
    achieved = alg_bytes / (part_avg * 1e-3) / 1e9
    peaks = _peaks()
    peak = peaks.get("hbm_gbs") or 6650.0
    # end to end through the public API with pinned host buffers: every
    # turn copies the beam in, tracks and copies it back (blond_engine_
    # track_host pipelines the copies in chunks against the particle pass)
    hdt = beam.dt.cpu().pin_memory()
    hdE = fused.dE.cpu().pin_memory()
    s = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    fused.track_host(hdt, hdE, 1, chunks=E2E_CHUNKS)  # warm-up: streams, events
    torch.cuda.synchronize()
    a.record(s)
    fused.track_host(hdt, hdE, E, chunks=E2E_CHUNKS)
    b.record(s)
    torch.cuda.synchronize()
    e2e_ms = a.elapsed_time(b)
    e2e_value = world * n * E / (dist_max(e2e_ms, world) * 1e-3)
    bytes_io = int(hdt.numel() * hdt.element_size() + hdE.numel() * hdE.element_size())
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": ms_max / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": args.precision, "data": "synthetic",
        "config": {"workload": WORKLOAD, "particles": n, "slices": S, "n_fft": n_fft,
                   "intensity": 1e10, "turns_per_graph": 50,
                   "autotuned": fused.tuned,
                   **({"beam_phase_loop": FEEDBACK_CONFIGS[args.feedback]}
                      if args.feedback != "none" else {}),
                   "l2": f"inputs larger than L2: {alg_bytes // 2 / 1e6:.0f} MB of dt/dE read per turn",
                   "parallelism": (f"dp{world}: one beam of {world} x {n:.0e} particles, "
                                   "int32 histogram all-reduce (NCCL) per turn")
                   if world > 1 else "1 GPU"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": _traffic(args.precision, n, fused.kernel),
                     "kernel": {"tma": "particle_kernel_tma", "stab": "particle_kernel_stab",
                                "packed": "particle_kernel_stab<TAB_GLOBAL>"}
                               .get(fused.kernel, "particle_kernel") + " (lik+kick+drift+deposit)",
                     "kernel_ms": part_avg, "head_kernel_ms": head_avg,
                     # the head's share of a graph-replayed turn: the turn
                     # minus the particle pass's own event-timed launch
                     "head_exposed_ms": max(0.0, ms_max / K - part_avg),
                     "turn_frac": alg_bytes / (ms_max / K * 1e-3) / 1e9 / peak,
                     "bytes_per_particle": BYTES_PER_PARTICLE[args.precision],
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (burst copy)"
                     if peaks.get("hbm_gbs") else "fallback 6650 GB/s"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": bytes_io,
                "d2h_bytes_per_step": bytes_io,
                "note": f"per turn: pinned H2D of dt+dE, one fused turn, D2H of dt+dE, "
                        f"pipelined in {E2E_CHUNKS} chunks (blond_engine_track_host)"},
        "gpu_launches": 2 * K,
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_mixed and args.precision == "f64":
        del fused, beam
        torch.cuda.empty_cache()
        for prec, key in (("f32p64", "mixed_precision"), ("q32p64", "fixed_point")):
            fm, bm_, _ = build_fused(n, S, W + K + kt + 4, prec, args.kernel, shape=shape)
            fm.track(W)
            fm.prepare()
            ms32 = time_turns(fm, K)
            h32, p32 = fm.time_kernels(kt)
            fm.check()
            ach32 = BYTES_PER_PARTICLE[prec] * n / (p32 / kt * 1e-3) / 1e9
            out[key] = {"dtype": prec, "value": n * K / (ms32 * 1e-3),
                        "ms_per_step": ms32 / K, "kernel_ms": p32 / kt,
                        "head_kernel_ms": h32 / kt,
                        "achieved_gbs": ach32, "frac": ach32 / peak,
                        "autotuned": fm.tuned}
            del fm, bm_
            torch.cuda.empty_cache()
    if rank == 0 and world == 1 and not args.no_batched:
        if "fused" in locals():
            del fused, beam
        torch.cuda.empty_cache()
        T = max(args.batched_error_turns, W + K)
        m = c3_measure(256, W, K, T, controls=("shift",))
        q, f32, f64 = (m["runs"][k] for k in ("q32p64", "f32p64", "f64"))
        nt = m["n_total"]
        pp = q["autotuned"]["particle_pass_ms"]
        eq, ef = m["errors"]["q32p64"], m["errors"]["f32p64"]
        out["batched"] = {
            "workload": C3_WORKLOAD, "beams": 256, "particles_total": nt,
            "dtype": "q32p64", "value": q["value"], "unit": UNIT,
            "ms_per_step": q["ms_per_step"], "steps": K,
            "particle_pass_ms": pp,
            "achieved_gbs": 24 * nt / (pp * 1e-3) / 1e9,
            "frac": 24 * nt / (pp * 1e-3) / 1e9 / peak,
            "turn_level_gbs": 24 * nt / (q["ms_per_step"] * 1e-3) / 1e9,
            "ratio_to_plain_f64_value": q["value"] / value,
            "rel_err_turns": m["turns"],
            "rel_err_statistic": "in-window rms bunch length and energy spread per beam "
                                 "vs the FP64 batch",
            "beams_within_1e-5": int(np.sum(eq.max(axis=1) <= 1e-5)),
            "max_rel_err": float(eq.max()),
            "profile_l2_rel_err": _l2_summary(m["profile_l2"]["q32p64"]),
            "autotuned": q["autotuned"],
            "clocks": q["clocks"],
            "f32p64": {"value": f32["value"], "ms_per_step": f32["ms_per_step"],
                       "beams_within_1e-5": int(np.sum(ef.max(axis=1) <= 1e-5)),
                       "max_rel_err": float(ef.max()),
                       "profile_l2_rel_err": _l2_summary(m["profile_l2"]["f32p64"]),
                       "clocks": f32["clocks"]},
            "f64": {"value": f64["value"], "ms_per_step": f64["ms_per_step"]},
            "control_fp64_dE_plus_0.01eV": {
                "what": "FP64 from energies moved by 0.01 eV vs FP64: the beams' own "
                        "sensitivity after the same turns",
                "beams_within_1e-5": int(np.sum(m["controls"]["shift"].max(axis=1) <= 1e-5)),
                "max_rel_err": float(m["controls"]["shift"].max()),
                "profile_l2_rel_err": _l2_summary(m["profile_l2"]["control_shift"])},
        }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, turns, kind, cores, sec = cpu_reference(n, S, None, args.cpu_seconds)
        out["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": cores, "kind": kind,
                               "sample": f"{turns} turns of the full {n:.0e}-particle "
                                         f"workload ({sec:.1f} s)"}
    return out


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _traffic(precision, n, kernel="plain"):
    """DRAM bytes per launch of the particle kernel from the committed ncu
    summary of that kernel (scaled to n particles), or None."""
    name = {"stab": "particle_kernel_stab_c2.txt", "plain": "particle_kernel_c2.txt",
            "packed": "particle_kernel_packed_c5_q32.txt"}.get(kernel)
    if precision == "q32p64" and kernel == "plain":
        name = "particle_kernel_q32_c2.txt"
    if name is None:
        return None
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.startswith(f"traffic_bytes_per_particle_{precision}:"):
                return float(line.split(":")[1]) * n
    except OSError:
        pass
    return None


# ----------------------------------------------------------------- ref arm
def gpu_reference(n: int, S: int, turns: int, warmup: int):
    """The reference's own GPU kernels (blond/gpu/kernels.cu rebuilt for
    sm_100a) + cuFFT, driven in the reference objects' order on device-
    resident coordinates; returns (particle-turns/s, ms per turn) or None
    when the kernels were not built or no GPU is present."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_cpu
    import ref_gpu
    import torch
    if not (ref_gpu.available() and torch.cuda.is_available()):
        return None
    ring, rf = machine(turns + warmup + 2)
    dt, dE, centre = host_bunch(ring, rf, n)
    cl, cr, bc = window(centre, S)
    bin_size = (cr - cl) / S
    Z = _resonator_host(ref_cpu.CpuPath(), np.fft.rfftfreq(S, bin_size)) / bin_size
    path = ref_gpu.RefGpuPath()
    path.setup(ref_cpu.programme(rf), turns + warmup)
    ddt, ddE = torch.tensor(dt, device="cuda"), torch.tensor(dE, device="cuda")
    prof = torch.zeros(S, dtype=torch.float64, device="cuda")
    dbc = torch.tensor(bc, device="cuda")
    dZ = torch.tensor(Z, device="cuda")
    factor = torch.empty(2 * (S - 1), dtype=torch.float64, device="cuda")
    path.slice(ddt, prof, cl, cr)
    args = ((cl, cr), dbc, dZ, S, 1.0, 1e10 / n, factor)
    for t in range(warmup):
        path.turn(t, ddt, ddE, prof, *args)
    s = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(s)
    for t in range(warmup, warmup + turns):
        path.turn(t, ddt, ddE, prof, *args)
    b.record(s)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / turns
    return n / (ms * 1e-3), ms


def run_reference(args, world, rank):
    n = int(args.particles)
    W, K = max(3, args.warmup), args.steps
    v, turns, kind, cores, sec = cpu_reference(n, args.slices, K, None, warmup=W)
    g = gpu_reference(n, args.slices, K, W)
    extra = {} if g is None else {"reference_gpu_kernels": {
        "value": g[0], "unit": UNIT, "ms_per_step": g[1],
        "what": "the reference's blond/gpu/kernels.cu rebuilt for sm_100a as blond/compile.py "
                "builds it (--use_fast_math, -maxrregcount 32), 2 x SMs blocks of 1024 "
                "threads, cuFFT for the FFT step, device-resident coordinates, FP64"}}
    return {**extra,
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
        "steps": K, "warmup": W, "ms_per_step": sec / K * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "particles": n, "slices": args.slices,
                   "n_fft": args.slices, "intensity": 1e10,
                   "parallelism": f"{cores} host threads"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": f"{K} turns of the full workload after {W} warm-up"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_reference_c3(args):
    """The reference on the C3 batch: every beam through its own objects,
    one after the other -- on the GPU with the reference's kernels rebuilt
    for sm_100a (the plain FP64 GPU path), and a bounded CPU sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref_cpu
    import ref_gpu
    import torch
    W, K = 2, max(1, min(args.steps, 5))
    beams = c3_beams(args.beams, W + K + 4)
    n_total = sum(b.n_macroparticles for _, b, _, _ in beams)
    cpu = ref_cpu.CpuPath()
    S = 512
    items = []
    for rf, beam, prof, tiv in beams:
        iv = tiv.induced_voltage_list[0]
        res = iv.impedance_source_list[0]
        bs = float(prof.bin_size)
        Z = _resonator_host(cpu, np.fft.rfftfreq(iv.n_fft, bs), res.R_S, res.Q,
                            res.frequency_R) / bs
        items.append((rf, beam, prof, iv.n_fft, Z))
    out = {}
    if ref_gpu.available() and torch.cuda.is_available():
        path = ref_gpu.RefGpuPath()
        state = []
        for rf, beam, prof, n_fft, Z in items:
            dt = beam.dt.detach().to("cuda", torch.float64).clone()
            dE = beam.dE.detach().to("cuda", torch.float64).clone()
            p = torch.zeros(S, dtype=torch.float64, device="cuda")
            cuts = (float(prof.cut_left), float(prof.cut_right))
            path.slice(dt, p, *cuts)
            state.append((dt, dE, p, cuts, torch.tensor(np.asarray(prof.bin_centers),
                                                        device="cuda"),
                          torch.tensor(Z, device="cuda"), n_fft,
                          float(rf.particle.charge), float(beam.ratio),
                          torch.empty(2 * (S - 1), dtype=torch.float64, device="cuda"),
                          path.programme(ref_cpu.programme(rf))))

        def one_turn(t):
            for dt, dE, p, cuts, bc, Z, n_fft, q, ratio, fac, prog in state:
                path.turn(t, dt, dE, p, cuts, bc, Z, n_fft, q, ratio, fac, prog=prog)

        for t in range(W):
            one_turn(t)
        s = torch.cuda.current_stream()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(s)
        for t in range(W, W + K):
            one_turn(t)
        b.record(s)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / K
        out["reference_gpu_kernels"] = {
            "value": n_total / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms,
            "what": "every beam through the reference's GPU kernels (blond/gpu/kernels.cu "
                    "rebuilt for sm_100a) + cuFFT, beam after beam as its objects run, FP64"}
    # CPU: one turn of every beam
    sec = 0.0
    for rf, beam, prof, n_fft, Z in items:
        dt = beam.dt.detach().cpu().numpy().astype(np.float64).copy()
        dE = beam.dE.detach().cpu().numpy().astype(np.float64).copy()
        sec += cpu.run(dt, dE, ref_cpu.programme(rf), 1, 0, impedance=(n_fft, Z),
                       cuts=(float(prof.cut_left), float(prof.cut_right)),
                       bin_centers=np.asarray(prof.bin_centers), n_slices=S,
                       charge=float(rf.particle.charge), ratio=float(beam.ratio))
    v = n_total / sec
    return {
        **out, "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": 1,
        "steps": 1, "warmup": 0, "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": C3_WORKLOAD, "beams": args.beams, "particles_total": n_total,
                   "slices": S, "n_fft": S, "parallelism": f"{cpu.cores} host threads"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cpu.cores, "kind": cpu.kind,
                         "sample": "one turn of every beam"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


C3_WORKLOAD = ("256 independent beams, double RF h=4620/18480 V2/V1=0.1 phi2=pi, "
               "V1 ~ U(2,7) MV, N_b log-uniform in [1e5, 4e6], sigma_dt ~ U(0.2,0.5) ns, "
               "512 slices, 3 resonators (R 2e5/1e5/5e4 Ohm, f_r 0.2/0.8/1.4 GHz, "
               "Q log-uniform [100, 30000]), intensity 1e11 protons per beam")
C3_INTENSITY = 1e11


def c3_beams(n_beams, turns, seed=1234, scale_particles=1.0):
    """The C3 scan: drop-in objects of every beam (seeded)."""
    import torch
    from blond_b200.beam.beam import Beam, Proton
    from blond_b200.beam.distributions import _get_dE_from_dt, bigaussian_arrays
    from blond_b200.beam.profile import CutOptions, Profile
    from blond_b200.impedances.impedance import InducedVoltageFreq, TotalInducedVoltage
    from blond_b200.impedances.impedance_sources import Resonators
    from blond_b200.input_parameters.rf_parameters import RFStation
    from blond_b200.input_parameters.ring import Ring
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_beams):
        n = int(round(np.exp(rng.uniform(np.log(1e5), np.log(4e6))) * scale_particles))
        V1 = rng.uniform(2e6, 7e6)
        sdt = rng.uniform(0.2e-9, 0.5e-9)
        Q = np.exp(rng.uniform(np.log(100), np.log(30000), 3))
        ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), turns)
        rf = RFStation(ring, [4620, 4 * 4620], [V1, 0.1 * V1], [0.0, np.pi], n_rf=2)
        centre = (rf.phi_s[0] - rf.phi_rf[0, 0]) / rf.omega_rf[0, 0]
        dt, dE = bigaussian_arrays(n, sdt, _get_dE_from_dt(ring, rf, sdt), centre, seed + k)
        beam = Beam(ring, n, C3_INTENSITY, dt=dt, dE=dE, dtype=torch.float64)
        prof = Profile(beam, CutOptions(cut_left=centre - 1.25e-9,
                                        cut_right=centre + 1.25e-9, n_slices=512))
        iv = InducedVoltageFreq(beam, prof, [Resonators([2e5, 1e5, 5e4],
                                                        [200e6, 800e6, 1.4e9], Q)])
        out.append((rf, beam, prof, TotalInducedVoltage(beam, prof, [iv])))
    return out


def ct_stream():
    import ctypes
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _c3_rel_errs(beams, other, ref):
    """Per beam: relative error of the in-window rms bunch length and
    energy spread of `other` against `ref` (both BatchTrackers)."""
    out = []
    for k, (_, _, p, _) in enumerate(beams):
        x = (ref.coordinates(k)[0].cpu().numpy(), ref.energies(k).cpu().numpy())
        y = (other.coordinates(k)[0].cpu().numpy(), other.energies(k).cpu().numpy())
        w = (x[0] > p.cut_left) & (x[0] < p.cut_right)
        out.append([abs(np.std(v[w]) / np.std(u[w]) - 1) for u, v in zip(x, y)])
    return np.array(out)


def _c3_profile_l2(other, ref):
    """Per beam: ||p_other - p_ref||_2 / ||p_ref||_2 of the profiles (the
    turn's slice counts) of two BatchTrackers."""
    po, pr = other.profiles_tensor(), ref.profiles_tensor()
    return ((po - pr).norm(dim=1) / pr.norm(dim=1).clamp_min(1e-300)).cpu().numpy()


def _l2_summary(v):
    return {"median": float(np.median(v)), "p90": float(np.percentile(v, 90)),
            "max": float(v.max())}


def _err_summary(errs):
    return {"sigma_dt_median": float(np.median(errs[:, 0])),
            "sigma_dt_p90": float(np.percentile(errs[:, 0], 90)),
            "sigma_dt_max": float(errs[:, 0].max()),
            "sigma_dE_median": float(np.median(errs[:, 1])),
            "sigma_dE_p90": float(np.percentile(errs[:, 1], 90)),
            "sigma_dE_max": float(errs[:, 1].max()),
            "beams_within_1e-5": int(np.sum(errs.max(axis=1) <= 1e-5))}


def c3_measure(n_beams, W, K, T_err, precisions=("q32p64", "f32p64", "f64"),
               controls=("ulp", "shift"), unbatched=False, shape=None):
    """C3: every precision batched (autotuned launch shape, graph-replayed
    turns), timed over K turns after W, then tracked on (untimed) to turn
    T_err, where each form's per-beam rms errors against FP64 are taken.
    controls -- how far the dynamics alone separate two FP64 runs: "ulp",
    FP64 again from initial times moved by one ulp (no bin changes);
    "shift", FP64 from initial energies moved by 0.01 eV (1e-10 of the
    spread, ten times below the Q32P64 grid).  unbatched: every beam
    through its own FP64 engine, one after the other.  shape: a fixed
    launch shape (threads, blocks per SM, particles per thread, chunk)
    instead of the autotuner's."""
    import torch
    from blond_b200.batch import BatchTracker
    from blond_b200.engine import FusedTracker
    from blond_b200.trackers.tracker import RingAndRFTracker
    beams = c3_beams(n_beams, T_err + W + K + 4)
    n_total = sum(b.n_macroparticles for _, b, _, _ in beams)
    res, trackers = {}, {}
    for prec in precisions:
        bt = BatchTracker([(RingAndRFTracker(rf, b), p, t) for rf, b, p, t in beams],
                          precision=prec)
        if shape is None:
            picked = bt.autotune()
        else:
            bt.set_shape(*shape)
            picked = {"threads": shape[0], "blocks_per_sm": shape[1],
                      "particles_per_thread": shape[2], "chunk": shape[3],
                      "particle_pass_ms": None}
        bt.track(W)
        bt.prepare()
        clocks = ClockSampler(torch.cuda.current_device())
        ms = time_turns(bt, K)
        clk = clocks.stop()
        bt.track(T_err - W - K)  # untimed, to the comparison turn
        bt.check()
        res[prec] = {"value": n_total * K / (ms * 1e-3), "ms_per_step": ms / K,
                     "autotuned": picked, "clocks": clk}
        trackers[prec] = bt
        for rf, _, _, _ in beams:
            rf.counter[0] = 0
    out = {"n_total": n_total, "turns": T_err, "runs": res}
    if "f64" in trackers:
        for prec in precisions:
            if prec != "f64":
                out.setdefault("profile_l2", {})[prec] = _c3_profile_l2(trackers[prec],
                                                                       trackers["f64"])
                out.setdefault("errors", {})[prec] = _c3_rel_errs(
                    beams, trackers[prec], trackers["f64"])
        for ctl in controls:
            bp = BatchTracker([(RingAndRFTracker(rf, b), p, t) for rf, b, p, t in beams],
                              precision="f64")
            if ctl == "ulp":
                bp.dt.copy_(torch.nextafter(bp.dt, torch.full_like(bp.dt, float("inf"))))
            else:
                bp.dE.add_(0.01)
            bp._call("slice", ct_stream())
            bp.track(T_err)
            for rf, _, _, _ in beams:
                rf.counter[0] = 0
            out.setdefault("controls", {})[ctl] = _c3_rel_errs(beams, bp, trackers["f64"])
            out.setdefault("profile_l2", {})["control_" + ctl] = _c3_profile_l2(
                bp, trackers["f64"])
            del bp
    del trackers
    torch.cuda.empty_cache()
    if unbatched:
        engines = [FusedTracker(RingAndRFTracker(rf, b), p, t, precision="f64",
                                turns_per_graph=K) for rf, b, p, t in beams]
        for e in engines:
            e.track(W)
            e.prepare()
        torch.cuda.synchronize()
        s = torch.cuda.current_stream()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        for e in engines:
            e.track(K)
        b.record(s)
        torch.cuda.synchronize()
        ms_plain = a.elapsed_time(b)
        out["unbatched_f64"] = {"value": n_total * K / (ms_plain * 1e-3),
                                "ms_per_step": ms_plain / K}
    return out


C5_WORKLOAD = ("1e8 protons 26 GeV/c, double RF h=4620/18480 4.5/0.45 MV (phi 0/pi), "
               "2^16 slices over 2.5 ns, "
               "4 resonators (R 2e5/1e5/5e4/3e4 Ohm, f_r 0.2/0.8/1.4/2.0 GHz, "
               "Q 100/1000/3000/30000) + inductive Im(Z)/n 0.1 Ohm, intensity 1e11")


def build_c5(n, n_turns, precision, seed=0, shape=None, kernel="auto"):
    """The C5 pipeline: a long profile (2^16 slices, histogram deposited
    straight into global memory) and a sum of five impedance sources."""
    import torch
    from blond_b200.beam.beam import Beam
    from blond_b200.beam.profile import CutOptions, Profile
    from blond_b200.engine import FusedTracker
    from blond_b200.impedances.impedance import (InducedVoltageFreq, InductiveImpedance,
                                                 TotalInducedVoltage)
    from blond_b200.impedances.impedance_sources import Resonators
    from blond_b200.trackers.tracker import RingAndRFTracker
    from blond_b200.input_parameters.rf_parameters import RFStation
    ring, _ = machine(n_turns)
    rf = RFStation(ring, [4620, 4 * 4620], [4.5e6, 0.45e6], [0.0, np.pi], n_rf=2)
    dt, dE, centre = host_bunch(ring, rf, n, seed)
    beam = Beam(ring, n, 1e11, dt=dt, dE=dE, dtype=torch.float64)
    del dt, dE
    cl, cr, _ = window(centre, 65536)
    prof = Profile(beam, CutOptions(cut_left=cl, cut_right=cr, n_slices=65536))
    iv = InducedVoltageFreq(beam, prof, [Resonators([2e5, 1e5, 5e4, 3e4],
                                                    [200e6, 800e6, 1.4e9, 2.0e9],
                                                    [100.0, 1000.0, 3000.0, 30000.0])])
    ind = InductiveImpedance(beam, prof, [0.1] * (n_turns + 1), rf)
    tiv = TotalInducedVoltage(beam, prof, [iv, ind])
    if shape is None:
        fused = FusedTracker(RingAndRFTracker(rf, beam), prof, tiv, precision=precision,
                             turns_per_graph=50)
    else:
        threads, bps, ring_stages = shape
        fused = FusedTracker(RingAndRFTracker(rf, beam), prof, tiv, precision=precision,
                             turns_per_graph=50, kernel="packed" if kernel == "auto" else kernel,
                             threads=threads, blocks_per_sm=bps, tune="fixed")
        fused.eng.call("set_prefetch", ring_stages)
        fused.eng.call("set_overlap", 0)  # what the autotuner picks at 2^16 slices
    return fused, beam, prof, iv.n_fft


def run_c5(args):
    """Q32P64 (the chosen form), F32P64 and FP64 on the same bunch, and an
    FP64 control from energies moved by 0.01 eV; each form's error is the
    in-window rms of dt and dE after the timed turns, against FP64."""
    import torch
    W, K = max(3, args.warmup), args.steps
    kt = min(K, 20)
    n = int(args.particles) if args.particles != 1e7 else int(1e8)
    res, coords, profs = {}, {}, {}
    peak = _peaks().get("hbm_gbs") or 6650.0
    shape = ((args.threads, args.blocks_per_sm, args.prefetch) if args.tune == "fixed"
             else None)
    forms = args.c5_forms.split(",")
    for prec, shift in (("q32p64", 0.0), ("f32p64", 0.0), ("f64", 0.0), ("f64", 0.01)):
        key = prec if not shift else "control_fp64_dE_plus_0.01eV"
        if (key if not shift else "control") not in forms:
            continue
        fused, beam, prof, n_fft = build_c5(n, W + K + kt + 4, prec, shape=shape,
                                            kernel=args.kernel)
        if shift:
            fused.dE.add_(shift)
            fused.eng.call("slice", ct_stream())
        fused.track(W)
        fused.prepare()
        torch.cuda.synchronize()
        clocks = ClockSampler(0) if prec == "q32p64" else None
        ms = time_turns(fused, K)
        clk = clocks.stop() if clocks else None
        fused.check()
        w = (fused.dt > prof.cut_left) & (fused.dt < prof.cut_right)
        coords[key] = (fused.dt[w].std().item(), fused.energies()[w].std().item())
        profs[key] = fused.profile_tensor().double().cpu()
        if not shift:
            head_ms, part_ms = fused.time_kernels(kt)
            ach = BYTES_PER_PARTICLE[prec] * n / (part_ms / kt * 1e-3) / 1e9
            res[prec] = {"value": n * K / (ms * 1e-3), "ms_per_step": ms / K,
                         "kernel_ms": part_ms / kt, "head_kernel_ms": head_ms / kt,
                         "achieved_gbs": ach, "frac": ach / peak, "clocks": clk,
                         "kernel": fused.kernel, "autotuned": fused.tuned}
        del fused, beam, prof
        torch.cuda.empty_cache()

    def err(key):
        if key not in coords or "f64" not in coords:
            return None
        return {"sigma_dt": abs(coords[key][0] / coords["f64"][0] - 1),
                "sigma_dE": abs(coords[key][1] / coords["f64"][1] - 1),
                "profile_l2": float((profs[key] - profs["f64"]).norm()
                                    / profs["f64"].norm())}
    r = res["q32p64"]
    return {
        "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": 1,
        "steps": K, "warmup": W, "ms_per_step": r["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "q32p64", "data": "synthetic",
        "config": {"workload": C5_WORKLOAD, "particles": n, "slices": 65536,
                   "n_fft": n_fft, "l2": "inputs larger than L2"},
        "roofline": {"bound": "hbm", "achieved": r["achieved_gbs"], "peak": peak,
                     "unit": "GB/s", "frac": r["frac"],
                     "traffic": _traffic("q32p64", n, r["kernel"]),
                     "kernel": {"tma": "particle_kernel_tma", "stab": "particle_kernel_stab",
                                "packed": "particle_kernel_stab<TAB_GLOBAL>"}
                               .get(r["kernel"], "particle_kernel"),
                     "kernel_ms": r["kernel_ms"], "head_kernel_ms": r["head_kernel_ms"],
                     "bytes_per_particle": BYTES_PER_PARTICLE["q32p64"],
                     "autotuned": r["autotuned"]},
        **{p: {k: res[p][k] for k in ("value", "ms_per_step", "kernel_ms", "head_kernel_ms",
                                      "achieved_gbs", "frac", "kernel")}
           for p in ("f32p64", "f64") if p in res},
        "rel_err_after_turns": {
            "turns": W + K, "statistic": "in-window rms of dt and dE vs FP64; "
                                         "profile_l2 = ||p - p_FP64||_2 / ||p_FP64||_2",
            "q32p64": err("q32p64"), "f32p64": err("f32p64"),
            "control_fp64_dE_plus_0.01eV": err("control_fp64_dE_plus_0.01eV")},
        "gpu_launches": 2 * K,
        "clocks": r["clocks"],
    }


C4_WORKLOAD = ("adjoint: 2e6 protons 26 GeV/c, h=4620 4.5 MV, 1024 slices over 2.5 ns "
               "(cloud-in-cell), broadband resonator 1 MOhm/1 GHz/Q=1 at intensity 3e9, "
               "500 turns, checkpoints every 50; loss = RMS bunch length^2 (ns^2) + L2 "
               "profile mismatch to a 0.35 ns Gaussian; gradients w.r.t. V[500], "
               "phi[500], R_s, f_r, Q")


def run_c4(args):
    """Gradient throughput (forward + backward, particle-turns/s counted
    once per turn of the map) in F32P64 and FP64, and the F32P64 gradient
    against the FP64 one."""
    import torch
    from blond_b200.adjoint import AdjointTracker, bunch_loss, gaussian_target
    n, S, T = 2_000_000, 1024, 500
    ring, rf = machine(T)
    dt0, dE0, centre = host_bunch(ring, rf, n, seed=3)
    cl, cr = centre - 1.25e-9, centre + 1.25e-9
    W, K = max(3, min(args.warmup, 3)), max(1, min(args.steps, 5))
    out, grads = {}, {}
    for prec in ("f32p64", "f64"):
        tr = AdjointTracker(ring, rf, n, 3e9, cl, cr, S, T, precision=prec,
                            checkpoint_every=50)
        target = gaussian_target(S, cl, cr, centre, 0.35e-9)
        dtt = torch.tensor(dt0, device="cuda")
        dEt = torch.tensor(dE0, device="cuda")

        def step():
            V = torch.full((T, 1), 4.5e6, dtype=torch.float64, device="cuda",
                           requires_grad=True)
            P = torch.zeros(T, 1, dtype=torch.float64, device="cuda", requires_grad=True)
            R, fr, Q = (torch.tensor([x], dtype=torch.float64, device="cuda",
                                     requires_grad=True) for x in (1e6, 1e9, 1.0))
            _, _, p = tr(dtt, dEt, V, P, tr.impedance(R, fr, Q))
            L = bunch_loss(p, target, tr.bin_centers())
            L.backward()
            return [x.grad for x in (V, P, R, fr, Q)]

        for _ in range(W):
            step()
        torch.cuda.synchronize()
        s = torch.cuda.current_stream()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(K + 1)]
        ev[0].record(s)
        for i in range(K):
            g = step()
            ev[i + 1].record(s)
        torch.cuda.synchronize()
        per = [ev[i].elapsed_time(ev[i + 1]) for i in range(K)]
        ms = ev[0].elapsed_time(ev[K]) / K
        grads[prec] = [x.detach().cpu().numpy().ravel() for x in g]
        # the median guards the figure against a step held up on a shared host
        out[prec] = {"ms_per_gradient": ms, "value": n * T / (ms * 1e-3),
                     "ms_per_gradient_median": float(np.median(per)),
                     "ms_per_gradient_each": per}
        del tr
        torch.cuda.empty_cache()
    names = ("V", "phi", "R_s", "f_r", "Q")
    err = {k: float(np.abs(a_ - b_).max() / np.abs(b_).max())
           for k, a_, b_ in zip(names, grads["f32p64"], grads["f64"])}
    r = out["f32p64"]
    return {
        "metric": "particle-turns/s of the gradient (forward + adjoint) on 1 B200",
        "value": r["value"], "unit": UNIT, "n_gpus": 1, "steps": K, "warmup": W,
        "ms_per_step": r["ms_per_gradient"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32p64", "data": "synthetic",
        "config": {"workload": C4_WORKLOAD, "particles": n, "slices": S, "turns": T},
        "ms_per_gradient_median": r["ms_per_gradient_median"],
        "ms_per_gradient_each": r["ms_per_gradient_each"],
        "f64": out["f64"],
        "f32p64_gradient_vs_f64": {"statistic": "max|g32 - g64| / max|g64| per parameter "
                                                "after 500 turns", **err},
        "fd_check": "tests/test_gpu_adjoint.py: FP64 adjoint vs central differences "
                    "of the FP64 forward within 1e-4 at this size",
    }


MTW_WORKLOAD = ("InducedVoltageResonator multi-turn wake: 1e6 protons 26 GeV/c, "
                "h=4620 4.5 MV, 1024 slices over 2.5 ns, 4 resonators (R 1e6/5e5/2e5/1e9 "
                "Ohm, f_r 0.2/0.63/0.915/1.4 GHz, Q 150/500/3e4/5e7), "
                "time_decay_factor 0.01")
MTW_METRIC = "induced-voltage points x resonators per second"
MTW_UNIT = "points*resonators/s"


def build_mtw(n=1_000_000, S=1024):
    from blond_b200.beam.beam import Beam
    from blond_b200.beam.profile import CutOptions, Profile
    from blond_b200.impedances.impedance import (InducedVoltageResonator,
                                                 TotalInducedVoltage)
    from blond_b200.impedances.impedance_sources import Resonators
    ring, rf = machine(2000)
    dt, dE, centre = host_bunch(ring, rf, n)
    beam = Beam(ring, n, 1e11, dt=dt, dE=dE)
    cl, cr, _ = window(centre, S)
    prof = Profile(beam, CutOptions(cut_left=cl, cut_right=cr, n_slices=S))
    res = Resonators([1e6, 5e5, 2e5, 1e9], [200e6, 630e6, 915e6, 1.4e9],
                     [150.0, 500.0, 3e4, 5e7])
    ivr = InducedVoltageResonator(beam, prof, res, multi_turn_wake=True, rf_station=rf,
                                  time_decay_factor=0.01)
    return beam, prof, res, ivr, TotalInducedVoltage(beam, prof, [ivr])


def _timed_steps(step, K, flush):
    """Sum of per-step CUDA-event times on the current stream, the L2
    flushed (untimed) before every step."""
    import torch
    s = torch.cuda.current_stream()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(K)]
    torch.cuda.synchronize()
    for a, b in ev:
        flush.zero_()
        a.record(s)
        step()
        b.record(s)
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in ev)


def mtw_cpu_baseline(prof_host, bc, bin_size, N, t, res, ratio, seconds):
    """The reference's time x bin evaluation (oracle restatement of
    butils_wrap_python.py:656-790) on blocks of time points until
    `seconds` have passed; points x resonators per second, 1 thread."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import wakes_oracle as wo
    done, t0 = 0, time.perf_counter()
    block = 512
    while time.perf_counter() - t0 < seconds and done < len(t):
        wo.resonator_induced_voltage(prof_host, bc, bin_size, N, t[done:done + block],
                                     res.R_S, res.omega_R, res.Q, 1.0, ratio)
        done += block
    sec = time.perf_counter() - t0
    return done * len(res.R_S) / sec, done


def run_mtw(args):
    import torch
    from blond_b200 import bmath as bm
    W, K = max(3, args.warmup), args.steps
    beam, prof, res, ivr, tiv = build_mtw()
    n_time, n_res, S = int(ivr.n_time), int(ivr.n_resonators), int(prof.n_slices)
    units = n_time * n_res
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    for _ in range(W):
        tiv.induced_voltage_sum()
    clocks = ClockSampler(0)
    ms = _timed_steps(tiv.induced_voltage_sum, K, flush)
    clk = clocks.stop()
    # the two kernels alone (scan + evaluation), same arguments as the class
    from scipy.constants import e as e_charge
    scale = -beam.particle.charge * e_charge * beam.n_macroparticles * beam.ratio

    def kernels():
        bm.resonator_induced_voltage(prof.n_macroparticles, ivr._bc_dev, prof.bin_size,
                                     beam.n_macroparticles, ivr._time_dev, ivr.R,
                                     ivr.omega_r, ivr.Q, scale,
                                     tmp_matrix=ivr._tmp_matrix, workspace=ivr._workspace)
    for _ in range(3):
        kernels()
    # replayed from a CUDA graph, so that the events bracket the two
    # launches and not the host's argument marshalling
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        kernels()
        torch.cuda.synchronize()
        with torch.cuda.graph(graph):
            kernels()
    torch.cuda.current_stream().wait_stream(side)
    for _ in range(3):
        graph.replay()
    kms = _timed_steps(graph.replay, K, flush) / K
    # bytes one launch pair must move: time array in, voltage and per-mode
    # rows out, profile and bin centres in, the recurrence written and read
    algo = 8 * n_time * (2 + n_res) + 16 * S + 2 * 16 * S * n_res + 8 * S
    peak = _peaks().get("hbm_gbs") or 6650.0
    ach = algo / (kms * 1e-3) / 1e9
    # end to end: the profile from pinned host memory, the summed voltage back
    hp = torch.empty(S, dtype=torch.float64, pin_memory=True)
    hp.copy_(prof.n_macroparticles.cpu())
    hv = torch.empty(S, dtype=torch.float64, pin_memory=True)
    s = torch.cuda.current_stream()

    def e2e_step():
        prof.n_macroparticles.copy_(hp, non_blocking=True)
        tiv.induced_voltage_sum()
        hv.copy_(tiv.induced_voltage, non_blocking=True)
    e_ms = _timed_steps(e2e_step, K, flush)
    cpu_v, sample = (None, 0)
    if not args.no_cpu_baseline:
        cpu_v, sample = mtw_cpu_baseline(
            prof.n_macroparticles.cpu().numpy(), np.asarray(prof.bin_centers), prof.bin_size,
            beam.n_macroparticles, np.asarray(ivr.time_array), res, beam.ratio,
            min(args.cpu_seconds, 12.0))
    return {
        "metric": MTW_METRIC, "value": units * K / (ms * 1e-3), "unit": MTW_UNIT,
        "n_gpus": 1, "steps": K, "warmup": W, "ms_per_step": ms / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": MTW_WORKLOAD, "slices": S, "n_time": n_time,
                   "resonators": n_res, "turns_of_memory": n_time // S,
                   "l2": "flushed (256 MiB write) before every timed step"},
        "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                     "frac": ach / peak, "traffic": None,
                     "kernel": "resonator_scan_kernel + resonator_eval_kernel",
                     "kernel_ms": kms, "algorithmic_bytes_per_launch": algo,
                     "note": "the evaluation issues one FP64 sincos + exp per point and "
                             "resonator; its bound is FP64 issue, not HBM"},
        "cpu_baseline": None if cpu_v is None else {
            "value": cpu_v, "unit": MTW_UNIT, "cores": 1, "kind": "port",
            "sample": f"{sample} of the {n_time} time points, the reference's time x bin "
                      "sum (numpy)"},
        "e2e": {"value": units * K / (e_ms * 1e-3), "unit": MTW_UNIT,
                "h2d_bytes_per_step": 8 * S, "d2h_bytes_per_step": 8 * S},
        "gpu_launches": 2 * K,
        "clocks": clk,
    }


def run_reference_mtw(args):
    """The reference's InducedVoltageResonator arithmetic on the host (the
    time x bin sum of butils_wrap_python.py:656-790, restated in numpy),
    one bounded sample of time points per step."""
    import torch
    W, K = 0, max(1, min(args.steps, 3))
    beam, prof, res, ivr, tiv = build_mtw()
    n_time, n_res = int(ivr.n_time), int(ivr.n_resonators)
    args_cpu = (prof.n_macroparticles.cpu().numpy(), np.asarray(prof.bin_centers),
                prof.bin_size, beam.n_macroparticles, np.asarray(ivr.time_array), res,
                beam.ratio)
    del tiv, ivr
    torch.cuda.empty_cache()
    vals = [mtw_cpu_baseline(*args_cpu, min(args.cpu_seconds, 12.0) / K) for _ in range(K)]
    v = float(np.mean([x[0] for x in vals]))
    sample = vals[0][1]
    return {
        "impl": "reference", "metric": MTW_METRIC, "value": v, "unit": MTW_UNIT,
        "n_gpus": 1, "steps": K, "warmup": W, "ms_per_step": n_time * n_res / v * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": MTW_WORKLOAD, "slices": int(prof.n_slices), "n_time": n_time,
                   "resonators": n_res, "parallelism": "1 host thread (numpy)"},
        "cpu_baseline": {"value": v, "unit": MTW_UNIT, "cores": 1, "kind": "port",
                         "sample": f"{sample} time points per step, scaled to the full "
                                   f"{n_time}"},
        "e2e": {"value": v, "unit": MTW_UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def main():
    args = parse()
    if args.workload == "c4" and args.impl == "ours":
        print(json.dumps(run_c4(args)), flush=True)
        return
    if args.workload == "c5" and args.impl == "ours":
        print(json.dumps(run_c5(args)), flush=True)
        return
    if args.workload == "mtw" and args.impl == "ours":
        print(json.dumps(run_mtw(args)), flush=True)
        return
    if args.workload == "c3" and args.impl == "ours":
        W, K = max(3, args.warmup), args.steps
        forms = tuple(args.c3_forms.split(","))
        shape = ((args.threads, args.blocks_per_sm, args.particles_per_thread, args.chunk)
                 if args.tune == "fixed" else None)
        T_err = max(args.batched_error_turns, W + K) if args.batched_error_turns > 0 else W + K
        m = c3_measure(args.beams, W, K, T_err, precisions=forms,
                       controls=("ulp", "shift") if args.batched_error_turns > 0 else (),
                       unbatched="f64" in forms, shape=shape)
        q = m["runs"]["q32p64"]
        peak = _peaks().get("hbm_gbs") or 6650.0
        print(json.dumps({
            "metric": METRIC, "value": q["value"], "unit": UNIT, "n_gpus": 1,
            "steps": K, "warmup": W, "ms_per_step": q["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "q32p64", "data": "synthetic",
            "config": {"workload": C3_WORKLOAD, "beams": args.beams,
                       "particles_total": m["n_total"], "slices": 512, "n_fft": 512},
            "runs": {k: {**v, "particle_pass_gbs": (24 if k != "f64" else 32) * m["n_total"]
                         / (v["autotuned"]["particle_pass_ms"] * 1e-3) / 1e9
                         if v["autotuned"].get("particle_pass_ms") else None}
                     for k, v in m["runs"].items()},
            "hbm_peak_gbs": peak,
            "unbatched_plain_f64": m.get("unbatched_f64"),
            "speedup_q32p64_batched_vs_unbatched_f64":
                q["value"] / m["unbatched_f64"]["value"] if "unbatched_f64" in m else None,
            "rel_err_after_turns": {
                "turns": m["turns"],
                "statistic": "in-window rms of dt and dE, per beam, vs the FP64 batch",
                **{k: _err_summary(v) for k, v in m.get("errors", {}).items()},
                **({"control_fp64_one_ulp": _err_summary(m["controls"]["ulp"]),
                    "control_fp64_dE_plus_0.01eV": _err_summary(m["controls"]["shift"])}
                   if m.get("controls") else {})},
            "profile_l2_rel_err_after_turns": {
                "statistic": "||p - p_FP64||_2 / ||p_FP64||_2 of each beam's profile",
                **{k: _l2_summary(v) for k, v in m.get("profile_l2", {}).items()}},
            "gpu_launches": 2 * K,
        }), flush=True)
        return
    if args.impl == "reference":
        os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        if rank != 0:
            return
        if args.workload == "c3":
            print(json.dumps(run_reference_c3(args)), flush=True)
            return
        if args.workload == "mtw":
            print(json.dumps(run_reference_mtw(args)), flush=True)
            return
        print(json.dumps(run_reference(args, world, rank)), flush=True)
        return
    world, rank, local = dist_init(args)
    try:
        out = run_ours(args, world, rank, local)
        if rank == 0:
            print(json.dumps(out), flush=True)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
