"""ctypes binding of libblond_b200.so (the C ABI in include/blond_b200.h).

The library is loaded from the in-tree build (blond_b200/_build/).  There is
no fallback: if the library is missing or CUDA is unavailable every entry
point raises, so nothing silently runs on the CPU.
"""
from __future__ import annotations

import ctypes as ct
import os
import threading

from .build import LIB

_lock = threading.Lock()
_lib = None

c_i64 = ct.c_int64
c_int = ct.c_int
c_dbl = ct.c_double
c_flt = ct.c_float
c_ptr = ct.c_void_p

# status codes (include/blond_b200.h)
OK = 0
ERR_NAMES = {
    1: "invalid argument", 2: "size out of range", 3: "misaligned pointer",
    4: "CUDA error", 5: "unsupported", 6: "timeout", 7: "bad state",
    8: "fixed-point energy out of range",
}


class BlondB200Error(RuntimeError):
    """A libblond_b200 call returned a non-zero status."""

    def __init__(self, func: str, code: int, message: str):
        self.code = code
        super().__init__(f"{func}: {ERR_NAMES.get(code, code)}: {message}")


def _sig(real):
    """argtypes of the bmath-level entry points for a real type."""
    P = c_ptr
    return {
        "kick": [P, P, c_int, real, P, P, P, c_i64, real, P],
        "rf_volt_comp": [P, P, P, P, c_int, c_i64, P, P],
        "drift": [P, P, c_int] + [real] * 11 + [c_i64, P],
        "histogram": [P, P, real, real, c_int, c_i64, P],
        "smooth_histogram": [P, P, real, real, c_int, c_i64, P],
        "linear_interp_kick": [P, P, P, P, real, c_int, c_i64, real, P],
        "beam_phase": [P, P, real, real, real, real, c_int, P, P],
        "beam_phase_fast": [P, P, real, real, real, c_int, P, P],
        "beam_statistics": [P, P, P, c_i64, P, P, P, P],
        "cut_limits": [P, c_i64, c_dbl, P, P, P, P],
    }


_EXTRA = {
    "blond_fast_resonator_f64": [c_ptr] * 6 + [c_int, c_i64, c_ptr],
    "blond_rfft_f64": [c_ptr, c_i64, c_i64, c_ptr, c_ptr],
    "blond_irfft_f64": [c_ptr, c_i64, c_ptr, c_i64, c_ptr],
    "blond_induced_voltage_f64": [c_ptr, c_int, c_ptr, c_i64, c_dbl, c_ptr,
                                  c_i64, c_ptr],
    "blond_engine_create": [ct.POINTER(c_ptr), c_int, c_int, c_int, c_int],
    "blond_engine_destroy": [c_ptr],
    "blond_engine_set_rf": [c_ptr, c_i64, c_ptr, c_ptr, c_ptr, c_ptr, c_dbl],
    "blond_engine_set_drift": [c_ptr, c_dbl, c_dbl] + [c_ptr] * 9,
    "blond_engine_set_slicing": [c_ptr, c_dbl, c_dbl, c_ptr],
    "blond_engine_set_impedance": [c_ptr, c_i64, c_ptr, c_dbl],
    "blond_engine_set_inductive": [c_ptr, c_ptr, c_dbl],
    "blond_engine_bind_beam": [c_ptr, c_ptr, c_ptr, c_i64],
    "blond_engine_set_turn": [c_ptr, c_i64, c_ptr],
    "blond_engine_slice": [c_ptr, c_ptr],
    "blond_engine_run": [c_ptr, c_i64, c_ptr],
    "blond_engine_prepare": [c_ptr, c_ptr],
    "blond_engine_check": [c_ptr, c_ptr],
    "blond_engine_set_kernel": [c_ptr, c_int],
    "blond_batch_create": [ct.POINTER(c_ptr), c_int, c_int, c_int, c_int, c_int],
    "blond_batch_destroy": [c_ptr],
    "blond_batch_set_rf": [c_ptr, c_i64, c_ptr, c_ptr, c_ptr, c_ptr, c_dbl],
    "blond_batch_set_drift": [c_ptr, c_dbl, c_dbl] + [c_ptr] * 9,
    "blond_batch_set_slicing": [c_ptr, c_ptr, c_ptr, c_ptr],
    "blond_batch_set_impedance": [c_ptr, c_i64, c_ptr, c_ptr],
    "blond_batch_bind_beams": [c_ptr, c_ptr, c_ptr, c_ptr],
    "blond_batch_set_turn": [c_ptr, c_i64, c_ptr],
    "blond_batch_slice": [c_ptr, c_ptr],
    "blond_batch_run": [c_ptr, c_i64, c_ptr],
    "blond_batch_prepare": [c_ptr, c_ptr],
    "blond_batch_tune": [c_ptr, c_int],
    "blond_batch_get_profiles": [c_ptr, c_ptr, c_ptr],
    "blond_batch_get_induced_voltages": [c_ptr, c_ptr, c_ptr],
    "blond_batch_set_energy_units": [c_ptr, c_ptr],
    "blond_batch_check": [c_ptr, c_ptr],
    "blond_batch_set_shape": [c_ptr, c_int, c_int, c_int, c_int, c_int],
    "blond_batch_autotune": [c_ptr, c_int, c_ptr, ct.POINTER(c_int), ct.POINTER(c_dbl)],
    "blond_engine_bind_histogram": [c_ptr, c_ptr],
    "blond_engine_step": [c_ptr, c_int, c_ptr],
    "blond_engine_get_profile": [c_ptr, c_ptr, c_ptr],
    "blond_engine_get_induced_voltage": [c_ptr, c_ptr, c_ptr],
    "blond_engine_get_turn": [c_ptr, ct.POINTER(c_i64)],
    "blond_engine_set_energy_unit": [c_ptr, c_dbl],
    "blond_engine_set_interpolation": [c_ptr, c_int],
    "blond_engine_set_smooth": [c_ptr, c_int],
    "blond_engine_tune": [c_ptr, c_int, c_int, c_int],
    "blond_engine_set_histogram": [c_ptr, c_int],
    "blond_engine_set_prefetch": [c_ptr, c_int],
    "blond_engine_set_l2_prefetch": [c_ptr, c_int],
    "blond_engine_set_overlap": [c_ptr, c_int],
    "blond_engine_set_cluster": [c_ptr, c_int],
    "blond_engine_track_host": [c_ptr, c_ptr, c_ptr, c_i64, c_int, c_ptr],
    "blond_engine_autotune": [c_ptr, c_int, c_ptr, ct.POINTER(c_int), ct.POINTER(c_dbl)],
    "blond_engine_time_kernels": [c_ptr, c_i64, ct.POINTER(c_dbl),
                                  ct.POINTER(c_dbl), c_ptr],
    "blond_turn_f64_noalloc": [c_ptr, c_ptr, c_i64, c_int, c_dbl, c_ptr, c_ptr, c_ptr,
                               c_dbl, c_int] + [c_dbl] * 13 + [c_int, c_ptr, c_i64,
                                                              c_dbl, c_ptr, c_ptr,
                                                              c_ptr],
    "blond_adjoint_deposit": [c_ptr, c_i64, c_int, c_dbl, c_dbl, c_ptr, c_ptr],
    "blond_adjoint_forward_turn": [c_int, c_ptr, c_ptr, c_ptr, c_ptr, c_i64, c_int,
                                   c_ptr, c_ptr, c_ptr, c_dbl, c_dbl, c_dbl, c_ptr,
                                   c_int, c_dbl, c_dbl, c_ptr, c_ptr],
    "blond_adjoint_backward_turn": [c_ptr, c_ptr, c_i64, c_ptr, c_ptr, c_ptr, c_int,
                                    c_int, c_ptr, c_ptr, c_ptr, c_dbl, c_dbl, c_ptr,
                                    c_int, c_dbl, c_dbl, c_ptr, c_ptr, c_ptr],
    "blond_adjoint_spectral": [c_int, c_ptr, c_int, c_ptr, c_i64, c_dbl, c_ptr, c_ptr,
                               c_ptr, c_ptr],
    "blond_adjoint_forward_run": [c_int, c_ptr, c_ptr, c_i64, c_int, c_i64, c_ptr, c_ptr,
                                  c_ptr, c_ptr, c_ptr, c_dbl, c_ptr, c_i64, c_dbl, c_ptr,
                                  c_ptr, c_ptr, c_int, c_dbl, c_dbl, c_int, c_ptr, c_ptr,
                                  c_ptr],
    "blond_adjoint_backward_run": [c_int, c_i64, c_int, c_i64, c_ptr, c_ptr, c_ptr, c_ptr,
                                   c_ptr, c_dbl, c_ptr, c_i64, c_dbl, c_ptr, c_ptr, c_int,
                                   c_dbl, c_dbl, c_int, c_ptr, c_ptr, c_ptr, c_ptr, c_ptr,
                                   c_ptr, c_ptr, c_ptr, c_ptr, c_ptr, c_ptr, c_ptr],
    "blond_engine_set_feedback": [c_ptr, c_int, c_int, c_dbl, c_dbl, c_dbl, c_int, c_dbl,
                                  c_dbl, c_dbl, c_int, c_ptr, c_ptr, c_int, c_ptr],
    "blond_engine_get_feedback": [c_ptr, c_ptr, c_ptr, c_ptr, c_ptr, c_ptr],
    "blond_resonator_workspace_bytes": [c_int, c_int],
    "blond_resonator_induced_voltage_f64": [c_ptr, c_ptr, c_int, c_dbl, c_dbl, c_ptr,
                                            c_i64, c_ptr, c_ptr, c_ptr, c_int, c_dbl,
                                            c_ptr, c_ptr, c_ptr, c_i64, c_ptr],
    "blond_resonator_mtw_f64": [c_ptr, c_ptr, c_int, c_dbl, c_dbl, c_ptr, c_i64,
                                c_ptr, c_ptr, c_ptr, c_int, c_dbl, c_ptr, c_ptr, c_i64,
                                c_i64, c_ptr, c_ptr, c_i64, c_ptr],
    "blond_interp_f64": [c_ptr, c_i64, c_dbl, c_ptr, c_ptr, c_int, c_dbl, c_dbl,
                         c_int, c_ptr, c_ptr],
}

# entry points that return a value instead of a status
_RESTYPE = {"blond_resonator_workspace_bytes": c_i64}


def exported_symbols() -> list[str]:
    """Every entry point include/blond_b200.h declares."""
    names = ["blond_b200_last_error", "blond_b200_version",
             "blond_b200_max_smem_slices"]
    for suffix in ("f64", "f32"):
        names += [f"blond_{k}_{suffix}" for k in _sig(c_dbl)]
    return names + list(_EXTRA)


def load(path: str | None = None) -> ct.CDLL:
    """Load (once) and annotate the library.  Raises if it is not built."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = path or LIB
        if not os.path.exists(path):
            raise ImportError(
                f"{path} is not built; run `python -m blond_b200.build` "
                "(blond_b200 has no CPU fallback)")
        lib = ct.CDLL(path)
        lib.blond_b200_last_error.restype = ct.c_char_p
        lib.blond_b200_last_error.argtypes = []
        lib.blond_b200_version.restype = c_int
        lib.blond_b200_max_smem_slices.restype = c_int
        for suffix, real in (("f64", c_dbl), ("f32", c_flt)):
            for k, argt in _sig(real).items():
                f = getattr(lib, f"blond_{k}_{suffix}")
                f.argtypes = argt
                f.restype = c_int
        for k, argt in _EXTRA.items():
            f = getattr(lib, k)
            f.argtypes = argt
            f.restype = _RESTYPE.get(k, c_int)
        _lib = lib
        return lib


def call(name: str, *args) -> None:
    """Call an entry point and raise BlondB200Error on a non-zero status."""
    lib = load()
    rc = getattr(lib, name)(*args)
    if rc != OK:
        msg = lib.blond_b200_last_error().decode(errors="replace")
        raise BlondB200Error(name, rc, msg)
