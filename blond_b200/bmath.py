"""bmath-level hot-path functions on CUDA tensors.

Same names, argument order and in-place semantics as the reference backend
functions that ``blond.utils.bmath`` dispatches to
(blond/utils/butils_wrap_cpp.py:835-989, declared in
blond/utils/bmath_backends.py:155-181).  Particle arrays are torch CUDA
tensors (float64 for the 'double' precision, float32 for 'single') and are
modified in place; small parameter arrays may be numpy arrays, lists or
tensors.  Every call is asynchronous on torch's current CUDA stream.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import torch
from scipy.constants import e

from . import _lib

__all__ = [
    "kick", "drift", "slice_beam", "slice_smooth", "linear_interp_kick",
    "rf_volt_comp", "fast_resonator", "rfft", "irfft", "rfftfreq",
    "induced_voltage_1turn", "interp", "resonator_induced_voltage", "beam_phase",
    "beam_phase_fast", "beam_statistics",
    "resonator_induced_voltage_1_turn", "resonator_workspace",
    "precision", "use_precision", "B200Backend",
]

_SOLVERS = {"simple": 0, "legacy": 1, "exact": 2}


class _Precision:
    """Mirror of blond.utils.PrecisionClass (utils/__init__.py:18-55)."""

    def __init__(self):
        self.set("double")

    def set(self, p: str = "double"):
        if p in ("single", "s", "32", "float32", "float", "f"):
            self.str, self.real_t, self.torch_t = "single", np.float32, torch.float32
            self.complex_t, self.num = np.complex64, 1
        elif p in ("double", "d", "64", "float64"):
            self.str, self.real_t, self.torch_t = "double", np.float64, torch.float64
            self.complex_t, self.num = np.complex128, 2
        else:
            raise ValueError(f"{p=} is not recognized, use 'single' or 'double'")


precision = _Precision()


def use_precision(p: str = "double") -> None:
    precision.set(p)


def _stream() -> ct.c_void_p:
    return ct.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ptr(t: torch.Tensor) -> ct.c_void_p:
    return ct.c_void_p(t.data_ptr())


def _suffix(t: torch.Tensor) -> str:
    if t.dtype == torch.float64:
        return "f64"
    if t.dtype == torch.float32:
        return "f32"
    raise TypeError(f"particle arrays must be float64 or float32, got {t.dtype}")


def _check_particles(*arrays: torch.Tensor) -> None:
    dtype = None
    for a in arrays:
        if not isinstance(a, torch.Tensor) or not a.is_cuda:
            raise TypeError("particle arrays must be CUDA tensors (in-place update)")
        if not a.is_contiguous():
            raise ValueError("particle arrays must be contiguous")
        if dtype is not None and a.dtype != dtype:
            raise TypeError(f"dtype mismatch: {a.dtype} vs {dtype}")
        dtype = a.dtype
    _suffix(arrays[0])


def as_device(x, dtype: torch.dtype, device=None) -> torch.Tensor:
    """Small parameter array -> contiguous CUDA tensor of ``dtype``."""
    if device is None:
        device = torch.device("cuda", torch.cuda.current_device())
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(np.asarray(x, dtype=np.float64)),
                           device=device).to(dtype).contiguous()


def _real(t: torch.Tensor):
    return _lib.c_dbl if t.dtype == torch.float64 else _lib.c_flt


# --------------------------------------------------------------------- kick
def kick(dt, dE, voltage, omega_rf, phi_rf, charge, n_rf, acceleration_kick):
    """butils_wrap_cpp.kick (:863-898) -> cpp_routines/kick.cpp:16-35."""
    _check_particles(dt, dE)
    r = _real(dt)
    V = as_device(voltage, dt.dtype, dt.device)
    om = as_device(omega_rf, dt.dtype, dt.device)
    ph = as_device(phi_rf, dt.dtype, dt.device)
    _lib.call(f"blond_kick_{_suffix(dt)}", _ptr(dt), _ptr(dE), int(n_rf),
              r(float(charge)), _ptr(V), _ptr(om), _ptr(ph), dt.numel(),
              r(float(acceleration_kick)), _stream())


def rf_volt_comp(voltages, omega_rf, phi_rf, bin_centers):
    """butils_wrap_cpp.rf_volt_comp (:835-860): returns a new array."""
    bc = bin_centers if isinstance(bin_centers, torch.Tensor) else as_device(
        bin_centers, precision.torch_t)
    bc = bc.contiguous()
    out = torch.zeros_like(bc)
    V = as_device(voltages, bc.dtype, bc.device)
    om = as_device(omega_rf, bc.dtype, bc.device)
    ph = as_device(phi_rf, bc.dtype, bc.device)
    _lib.call(f"blond_rf_volt_comp_{_suffix(bc)}", _ptr(V), _ptr(om), _ptr(ph),
              _ptr(bc), int(V.numel()), bc.numel(), _ptr(out), _stream())
    return out


# -------------------------------------------------------------------- drift
def drift(dt, dE, solver, t_rev, length_ratio, alpha_order, eta_0, eta_1,
          eta_2, alpha_0, alpha_1, alpha_2, beta, energy):
    """butils_wrap_cpp.drift (:901-943) -> cpp_routines/drift.cpp:19-78."""
    _check_particles(dt, dE)
    if solver not in _SOLVERS:
        raise KeyError(solver)
    r = _real(dt)
    vals = [t_rev, length_ratio, alpha_order, eta_0, eta_1, eta_2, alpha_0,
            alpha_1, alpha_2, beta, energy]
    _lib.call(f"blond_drift_{_suffix(dt)}", _ptr(dt), _ptr(dE),
              _SOLVERS[solver], *[r(float(v)) for v in vals], dt.numel(),
              _stream())


# ------------------------------------------------------------------ slicing
def slice_beam(dt, profile, cut_left, cut_right):
    """butils_wrap_cpp.slice_beam (:971-984) -> histogram.cpp:22-73."""
    _check_particles(dt, profile)
    r = _real(dt)
    _lib.call(f"blond_histogram_{_suffix(dt)}", _ptr(dt), _ptr(profile),
              r(float(cut_left)), r(float(cut_right)), profile.numel(),
              dt.numel(), _stream())


def slice_smooth(dt, profile, cut_left, cut_right):
    """butils_wrap_cpp.slice_smooth (:987-999) -> histogram.cpp:75-132."""
    _check_particles(dt, profile)
    r = _real(dt)
    _lib.call(f"blond_smooth_histogram_{_suffix(dt)}", _ptr(dt), _ptr(profile),
              r(float(cut_left)), r(float(cut_right)), profile.numel(),
              dt.numel(), _stream())


# ------------------------------------------------------ interpolated kick
def linear_interp_kick(dt, dE, voltage, bin_centers, charge,
                       acceleration_kick):
    """butils_wrap_cpp.linear_interp_kick (:946-968)."""
    _check_particles(dt, dE)
    r = _real(dt)
    V = as_device(voltage, dt.dtype, dt.device)
    bc = as_device(bin_centers, dt.dtype, dt.device)
    _lib.call(f"blond_linear_interp_kick_{_suffix(dt)}", _ptr(dt), _ptr(dE),
              _ptr(V), _ptr(bc), r(float(charge)), bc.numel(), dt.numel(),
              r(float(acceleration_kick)), _stream())


# ------------------------------------------------------- impedance / FFT
def fast_resonator(R_S, Q, frequency_array, frequency_R, impedance=None):
    """butils_wrap_cpp.fast_resonator (:1133-1171): complex128 tensor."""
    f = as_device(frequency_array, torch.float64)
    R = as_device(R_S, torch.float64)
    q = as_device(Q, torch.float64)
    fr = as_device(frequency_R, torch.float64)
    re = torch.zeros_like(f)
    im = torch.zeros_like(f)
    _lib.call("blond_fast_resonator_f64", _ptr(re), _ptr(im), _ptr(f), _ptr(R),
              _ptr(q), _ptr(fr), int(R.numel()), f.numel(), _stream())
    out = torch.complex(re, im)
    if impedance is not None and isinstance(impedance, torch.Tensor) and \
            impedance.dtype == torch.complex128 and impedance.numel() == out.numel():
        impedance.copy_(out)
        return impedance
    return out


def rfft(a, n=None):
    """numpy.fft.rfft(a, n) semantics (bmath_backends.py:447) in float64."""
    x = as_device(a, torch.float64).reshape(-1)
    n = int(x.numel() if n is None else n)
    out = torch.empty(n // 2 + 1, dtype=torch.complex128, device=x.device)
    _lib.call("blond_rfft_f64", _ptr(x), x.numel(), n, _ptr(out), _stream())
    return out


def irfft(a, n=None):
    """numpy.fft.irfft(a, n) semantics (bmath_backends.py:448) in float64."""
    if isinstance(a, torch.Tensor):
        spec = a.to(torch.complex128)
    else:
        spec = torch.as_tensor(np.asarray(a, dtype=np.complex128),
                               device=torch.device("cuda", torch.cuda.current_device()))
    spec = spec.reshape(-1).contiguous()
    m = spec.numel()
    n = int(2 * (m - 1) if n is None else n)
    need = n // 2 + 1
    if m < need:
        spec = torch.cat([spec, spec.new_zeros(need - m)])
    elif m > need:
        spec = spec[:need].contiguous()
    out = torch.empty(n, dtype=torch.float64, device=spec.device)
    _lib.call("blond_irfft_f64", _ptr(spec), n, _ptr(out), n, _stream())
    return out


def rfftfreq(n, d=1.0):
    """numpy.fft.rfftfreq (host arithmetic, setup only)."""
    return np.fft.rfftfreq(int(n), d)


def induced_voltage_1turn(profile, total_impedance, n_fft, scale, n_out):
    """-scale * irfft(total_impedance * rfft(profile, n_fft))[:n_out]
    (impedance.py:475-489) in one launch; float64 tensor of n_out values."""
    p = as_device(profile, torch.float64)
    Z = total_impedance if isinstance(total_impedance, torch.Tensor) else \
        torch.as_tensor(np.asarray(total_impedance, np.complex128),
                        device=p.device)
    Z = Z.to(torch.complex128).contiguous()
    out = torch.empty(int(n_out), dtype=torch.float64, device=p.device)
    _lib.call("blond_induced_voltage_f64", _ptr(p), p.numel(), _ptr(Z),
              int(n_fft), float(scale), _ptr(out), int(n_out), _stream())
    return out


# ------------------------------------------------------------ beam phase
def _beam_phase_call(name, bin_centers, profile, args, start=0, stop=None):
    p = profile
    if not isinstance(p, torch.Tensor):
        p = as_device(p, precision.torch_t)
    bc = as_device(bin_centers, p.dtype, p.device)
    stop = bc.numel() if stop is None else int(stop)
    start = int(start)
    if stop <= start:
        return float("nan")
    bcs, ps = bc[start:stop].contiguous(), p[start:stop].contiguous()
    out = torch.empty(1, dtype=p.dtype, device=p.device)
    r = _real(p)
    _lib.call(f"{name}_{_suffix(p)}", _ptr(bcs), _ptr(ps), *[r(float(a)) for a in args],
              stop - start, _ptr(out), _stream())
    return out


def beam_phase(bin_centers, profile, alpha, omega_rf, phi_rf, bin_size, *,
               start=0, stop=None, device_result=False):
    """butils_wrap_cpp.beam_phase (:785-808): the beam phase coefficient
    (cpp_routines/beam_phase.cpp:6-40) of profile[start:stop], a float
    (NaN for an empty range).  device_result=True returns the one-element
    device tensor instead (no synchronisation)."""
    out = _beam_phase_call("blond_beam_phase", bin_centers, profile,
                           (alpha, omega_rf, phi_rf, bin_size), start, stop)
    if device_result or not isinstance(out, torch.Tensor):
        return out
    return float(out.item())


def beam_phase_fast(bin_centers, profile, omega_rf, phi_rf, bin_size, *,
                    start=0, stop=None, device_result=False):
    """butils_wrap_cpp.beam_phase_fast (:811-832), without the exp weight."""
    out = _beam_phase_call("blond_beam_phase_fast", bin_centers, profile,
                           (omega_rf, phi_rf, bin_size), start, stop)
    if device_result or not isinstance(out, torch.Tensor):
        return out
    return float(out.item())


# ------------------------------------------------------------ statistics
STATS_SCRATCH = 7 * 1024  # BLOND_STATS_SCRATCH


def beam_statistics(dt, dE, id=None, out=None, scratch=None, ticket=None):
    """Beam.statistics (beam.py:430-458) on the device: an 8-element float64
    tensor [n_alive, mean_dt, sigma_dt, mean_dE, sigma_dE, epsn_rms_l,
    sum dt^2, sum dE^2] over the particles with id != 0.  No
    synchronisation; pass the same out / scratch / ticket every call to
    reuse them (out carries the previous means as the sums' shift)."""
    if dt.dtype != dE.dtype:
        raise TypeError("dt and dE must have the same dtype")
    dev = dt.device
    if out is None:
        out = torch.full((8,), float("nan"), dtype=torch.float64, device=dev)
    if scratch is None:
        scratch = torch.empty(STATS_SCRATCH, dtype=torch.float64, device=dev)
    if ticket is None:
        ticket = torch.zeros(1, dtype=torch.int32, device=dev)
    idp = None
    if id is not None:
        id = id.to(torch.int64).contiguous()
        idp = _ptr(id)
    _lib.call(f"blond_beam_statistics_{_suffix(dt)}", _ptr(dt), _ptr(dE), idp, dt.numel(),
              _ptr(out), _ptr(scratch), _ptr(ticket), _stream())
    return out


def cut_limits(dt, n_sigma=None, scratch=None, ticket=None):
    """The automatic frame of CutOptions.set_cuts (profile.py:185-195) by a
    device reduction: a float64 device tensor [cut_left, cut_right] --
    min/max -/+ 5 % of the spread when n_sigma is None (the reference's
    bits), else mean -/+ n_sigma sigma / 2.  No synchronisation."""
    dev = dt.device
    if scratch is None:
        scratch = torch.empty(STATS_SCRATCH, dtype=torch.float64, device=dev)
    if ticket is None:
        ticket = torch.zeros(1, dtype=torch.int32, device=dev)
    out = torch.empty(2, dtype=torch.float64, device=dev)
    dt = dt.contiguous()
    _lib.call(f"blond_cut_limits_{_suffix(dt)}", _ptr(dt), dt.numel(),
              float(n_sigma) if n_sigma is not None else 0.0, _ptr(out), _ptr(scratch),
              _ptr(ticket), _stream())
    return out


# ------------------------------------------------------ time-domain wakes
def interp(x, xp, fp, left=None, right=None, period=None, *, x_shift=0.0):
    """numpy.interp(x + x_shift, xp, fp, left, right) on the device in
    float64 (bm.interp, bmath_backends.py:373); a tensor shaped like x.
    xp must be increasing, as numpy requires; ``period`` is not supported."""
    if period is not None:
        raise NotImplementedError("interp: period")
    X = as_device(x, torch.float64)
    shape = X.shape
    X = X.reshape(-1).contiguous()
    XP = as_device(xp, torch.float64, X.device).reshape(-1).contiguous()
    FP = as_device(fp, torch.float64, X.device).reshape(-1).contiguous()
    if XP.numel() == 0:
        raise ValueError("array of sample points is empty")
    if XP.numel() != FP.numel():
        raise ValueError("fp and xp are not of the same length.")
    out = torch.empty_like(X)
    flags = (1 if left is not None else 0) | (2 if right is not None else 0)
    _lib.call("blond_interp_f64", _ptr(X), X.numel(), float(x_shift), _ptr(XP),
              _ptr(FP), XP.numel(), float(0.0 if left is None else left),
              float(0.0 if right is None else right), flags, _ptr(out), _stream())
    return out.reshape(shape)


def resonator_workspace(n_slices: int, n_resonators: int, device=None):
    """Scratch for resonator_induced_voltage (uint8 device tensor)."""
    n = int(_lib.load().blond_resonator_workspace_bytes(int(n_slices),
                                                        int(n_resonators)))
    return torch.empty(n, dtype=torch.uint8, device=device or "cuda")


def resonator_induced_voltage(profile, bin_centers, bin_size, beam_n_macroparticles,
                              time_array, R, omega_r, Q, scale, out=None,
                              tmp_matrix=None, workspace=None, memory_in=None, shift=0):
    """Induced voltage of resonators by the analytic convolution of the
    linearly interpolated line density (butils_wrap_python.py:656-790),
    float64, one value per time_array point.  ``bin_centers`` must be
    increasing; R, omega_r, Q are host sequences; ``scale`` is
    -charge * e * beam_n_macroparticles * ratio.  ``tmp_matrix`` (optional,
    n_resonators x n_time float64 tensor) receives the per-resonator rows;
    ``workspace`` (from resonator_workspace) may be reused across calls.
    With ``memory_in`` (float64 device tensor of n_memory >= n_time points)
    the result is instead the next multi-turn memory, memory_in moved
    forward by ``shift`` points (zeros behind) plus the voltage on its first
    n_time points (impedance.py:1317-1335), n_memory values.
    Returns (induced_voltage or memory, workspace)."""
    p = as_device(profile, torch.float64).reshape(-1).contiguous()
    bc = as_device(bin_centers, torch.float64, p.device).reshape(-1).contiguous()
    t = as_device(time_array, torch.float64, p.device).reshape(-1).contiguous()
    Rh = np.ascontiguousarray(np.asarray(R, dtype=np.float64).reshape(-1))
    wh = np.ascontiguousarray(np.asarray(omega_r, dtype=np.float64).reshape(-1))
    qh = np.ascontiguousarray(np.asarray(Q, dtype=np.float64).reshape(-1))
    n_res = Rh.size
    if not (wh.size == qh.size == n_res):
        raise ValueError("R, omega_r and Q differ in length")
    if p.numel() != bc.numel():
        raise ValueError("profile and bin_centers differ in length")
    if workspace is None:
        workspace = resonator_workspace(bc.numel(), n_res, p.device)
    P = lambda a: a.ctypes.data_as(ct.c_void_p)  # noqa: E731
    tm = _ptr(tmp_matrix) if tmp_matrix is not None else None
    if memory_in is not None:
        mem = memory_in
        if mem.dtype != torch.float64 or not mem.is_contiguous():
            raise ValueError("memory_in must be a contiguous float64 tensor")
        if out is None:
            out = torch.empty_like(mem)
        _lib.call("blond_resonator_mtw_f64", _ptr(p), _ptr(bc), bc.numel(),
                  float(bin_size), float(beam_n_macroparticles), _ptr(t), t.numel(),
                  P(Rh), P(wh), P(qh), n_res, float(scale), _ptr(mem), _ptr(out),
                  mem.numel(), int(shift), tm, _ptr(workspace), workspace.numel(),
                  _stream())
        return out, workspace
    if out is None:
        out = torch.empty(t.numel(), dtype=torch.float64, device=p.device)
    _lib.call("blond_resonator_induced_voltage_f64", _ptr(p), _ptr(bc), bc.numel(),
              float(bin_size), float(beam_n_macroparticles), _ptr(t), t.numel(),
              P(Rh), P(wh), P(qh), n_res, float(scale), _ptr(out), tm,
              _ptr(workspace), workspace.numel(), _stream())
    return out, workspace


def resonator_induced_voltage_1_turn(kappa1, n_macroparticles, bin_centers, bin_size,
                                     n_time, deltaT, tArray, reOmegaP, imOmegaP,
                                     Qtilde, n_resonators, omega_r, Q, tmp_matrix,
                                     charge, beam_n_macroparticles, ratio, R,
                                     induced_voltage, float_precision):
    """butils_wrap_python.resonator_induced_voltage_1_turn (:656-790) with its
    signature; returns (induced_voltage, deltaT).  reOmegaP, imOmegaP and
    Qtilde are re-derived from omega_r and Q by the reference's formulas.
    kappa1 and tmp_matrix are filled when they are device tensors of the
    reference's shapes; deltaT, the n_time x n_slices matrix the reference
    builds, is only filled when it is such a tensor (the kernel never needs
    it)."""
    bc = as_device(bin_centers, torch.float64)
    if bc.numel() > 1 and not bool(torch.all(bc[1:] > bc[:-1])):
        raise ValueError("bin_centers must be increasing")
    t = as_device(tArray, torch.float64, bc.device).reshape(-1)[: int(n_time)]
    tm = None
    if isinstance(tmp_matrix, torch.Tensor) and tmp_matrix.dtype == torch.float64 \
            and tmp_matrix.is_contiguous() \
            and tuple(tmp_matrix.shape) == (int(n_resonators), t.numel()):
        tm = tmp_matrix
    scale = -charge * e * beam_n_macroparticles * ratio
    v, ws = resonator_induced_voltage(n_macroparticles, bc, bin_size,
                                      beam_n_macroparticles, t, R, omega_r, Q,
                                      scale, tmp_matrix=tm)
    if isinstance(kappa1, torch.Tensor) and kappa1.numel() == bc.numel() - 1:
        n_res = np.asarray(R).size
        off = n_res * bc.numel() * 16
        kappa1.copy_(ws[off: off + 8 * (bc.numel() - 1)].view(torch.float64))
    if isinstance(deltaT, torch.Tensor) and tuple(deltaT.shape) == (t.numel(), bc.numel()):
        torch.sub(t[:, None], bc[None, :], out=deltaT)
    dtype = torch.float32 if np.dtype(float_precision) == np.float32 else torch.float64
    v = v.to(dtype)
    if isinstance(induced_voltage, torch.Tensor) and induced_voltage.shape == v.shape \
            and induced_voltage.dtype == dtype:
        induced_voltage.copy_(v)
        v = induced_voltage
    return v, deltaT


def not_implemented(*args, **kwargs):
    """Stands in for an attribute of the backend contract this library does
    not provide (the reference's GpuBackend does the same for its gaps,
    bmath_backends.py:750-759)."""
    raise NotImplementedError("not provided by the B200 backend (outside the "
                              "tracking hot path)")


# Every attribute the reference's backend contract declares
# (MasterBackend.__init__, bmath_backends.py:61-185), in its order.
MASTER_ATTRIBUTES = (
    "precision", "device", "histogram2d", "maximum", "minimum", "amax", "roll",
    "fftconvolve", "pi", "diff", "uint", "empty", "sign", "vectorize", "hstack",
    "arctan", "arcsin", "sqrt", "trapezoid", "reshape", "exp", "int32", "delete",
    "unique", "abs", "zeros", "floor", "resize", "take", "round", "fabs", "float64",
    "meshgrid", "mean", "append", "argmax", "dot", "double", "sum", "cumsum", "cos",
    "concatenate", "full", "asarray", "ones", "uint32", "histogram", "unwrap", "ceil",
    "interp", "std", "empty_like", "min", "max", "cosh", "linspace", "array",
    "gradient", "isnan", "hamming", "clip", "where", "isinf", "sin", "zeros_like",
    "arange", "loadtxt", "convolve", "fliplr", "log", "heaviside", "absolute",
    "float32", "ascontiguousarray", "complex64", "copy", "poly1d", "invert", "all",
    "int64", "count_nonzero", "nonzero", "log10", "real", "argsort", "complex128",
    "irfft", "rfft", "rfftfreq", "random", "fft", "slice_beam", "drift",
    "sparse_histogram", "distribution_from_tomoscope", "set_random_seed",
    "synchrotron_radiation_full", "kick", "fast_resonator", "beam_phase_fast",
    "rf_volt_comp", "slice_smooth", "linear_interp_kick", "music_track_multiturn",
    "music_track", "synchrotron_radiation", "beam_phase",
    "resonator_induced_voltage_1_turn",
)


class B200Backend:
    """A complete backend for the reference's bmath object: every attribute
    of its contract (MasterBackend, bmath_backends.py:61-201) is set, so
    the reference's verify_backend (:203-228) accepts it.  As the
    reference's GpuBackend works on CuPy arrays, this one works on torch
    CUDA tensors: the hot-path routines are libblond_b200's kernels, the
    array functions torch's CUDA equivalents of the numpy names, and the
    routines outside the tracking hot path (synchrotron radiation, MuSiC,
    tomoscope import, sparse slicing) raise NotImplementedError."""

    def __init__(self):
        T = torch
        self.precision = precision
        self.device = "GPU_B200"
        # hot path: libblond_b200
        self.kick = kick
        self.drift = drift
        self.slice_beam = slice_beam
        self.slice_smooth = slice_smooth
        self.linear_interp_kick = linear_interp_kick
        self.rf_volt_comp = rf_volt_comp
        self.fast_resonator = fast_resonator
        self.rfft = rfft
        self.irfft = irfft
        self.rfftfreq = rfftfreq
        self.interp = interp
        self.beam_phase = beam_phase
        self.beam_phase_fast = beam_phase_fast
        self.resonator_induced_voltage_1_turn = resonator_induced_voltage_1_turn
        # array functions on CUDA tensors
        for name in ("maximum", "minimum", "amax", "roll", "diff", "empty", "sign",
                     "hstack", "arctan", "arcsin", "sqrt", "trapezoid", "reshape", "exp",
                     "unique", "abs", "zeros", "floor", "take", "round", "meshgrid", "mean",
                     "argmax", "dot", "sum", "cumsum", "cos", "concatenate", "full", "asarray",
                     "ones", "ceil", "std", "empty_like", "min", "max", "cosh", "linspace",
                     "gradient", "isnan", "clip", "where", "isinf", "sin", "zeros_like",
                     "arange", "fliplr", "log", "heaviside", "absolute", "all",
                     "count_nonzero", "nonzero", "log10", "real", "argsort", "histogram"):
            setattr(self, name, getattr(T, name))
        self.fabs = T.abs
        self.array = T.tensor
        self.copy = T.clone
        self.invert = T.bitwise_not
        self.hamming = T.hamming_window
        self.ascontiguousarray = lambda a, dtype=None: (
            T.as_tensor(a, dtype=dtype).contiguous())
        self.append = lambda a, b: T.cat([T.as_tensor(a).reshape(-1),
                                          T.as_tensor(b).reshape(-1)])
        self.pi = float(np.pi)
        for name, dt in (("int32", T.int32), ("int64", T.int64), ("uint32", T.uint32),
                         ("uint", T.uint64), ("float32", T.float32), ("float64", T.float64),
                         ("double", T.float64), ("complex64", T.complex64),
                         ("complex128", T.complex128)):
            setattr(self, name, dt)
        self.fft = T.fft
        self.random = T.random
        self.set_random_seed = T.manual_seed
        # outside the hot path
        for name in ("histogram2d", "fftconvolve", "vectorize", "delete", "resize",
                     "unwrap", "loadtxt", "convolve", "poly1d", "sparse_histogram",
                     "distribution_from_tomoscope", "synchrotron_radiation_full",
                     "synchrotron_radiation", "music_track_multiturn", "music_track"):
            setattr(self, name, not_implemented)

    def use_precision(self, p: str = "double"):
        use_precision(p)
