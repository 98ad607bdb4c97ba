"""REFERENCE GPU BASELINE DRIVER -- test/benchmark infrastructure, not product code.

Runs the reference's own GPU kernels (blond/gpu/kernels.cu, rebuilt for
sm_100a by oracle/Makefile as the reference builds them, launched by
oracle/_ref/libref_gpu_shim.so with the reference's launch geometry) in
the call sequence of the reference objects on its GPU backend:
TotalInducedVoltage.track (rfft -> x Z -> irfft with cuFFT, as CuPy does
for bmath_backends.py's GPU mapping; then linear_interp_kick =
lik_only_gm_copy + lik_only_gm_comp, butils_wrap_cupy.py:194-254) ->
RingAndRFTracker.track (simple_kick, drift; butils_wrap_cupy.py:69-191) ->
Profile.track (fill 0 + sm_histogram / hybrid_histogram,
butils_wrap_cupy.py:257-309).  Arrays are torch CUDA float64 tensors on
the current stream.  Differences from the reference's own driver: the
lik scratch is allocated once instead of per call, and there is no Python
object overhead per turn (both favour the reference).
"""
from __future__ import annotations

import ctypes as ct
import os

import torch
from scipy.constants import e as E_CHARGE

HERE = os.path.dirname(os.path.abspath(__file__))
SHIM = os.path.join(HERE, "_ref", "libref_gpu_shim.so")
CUBIN = os.path.join(HERE, "_ref", "kernels_sm_100a_double.cubin")


def available() -> bool:
    return os.path.exists(SHIM) and os.path.exists(CUBIN)


class RefGpuPath:
    def __init__(self):
        if not available():
            raise FileNotFoundError("reference GPU kernels not built (make -C oracle refgpu)")
        torch.cuda.init()
        torch.zeros(1, device="cuda")  # the primary context exists and is current
        self.lib = ct.CDLL(SHIM)
        self.lib.refgpu_error.restype = ct.c_char_p
        P, I, D = ct.c_void_p, ct.c_int, ct.c_double
        self.lib.refgpu_load.argtypes = [ct.c_char_p]
        self.lib.refgpu_kick.argtypes = [P, P, I, D, P, P, P, I, D, P]
        self.lib.refgpu_drift.argtypes = [P, P, I] + [D] * 11 + [I, P]
        self.lib.refgpu_slice.argtypes = [P, P, D, D, ct.c_uint, I, P]
        self.lib.refgpu_lik.argtypes = [P, P, P, P, D, I, I, D, P, P]
        self._check(self.lib.refgpu_load(CUBIN.encode()))

    def _check(self, rc):
        if rc:
            raise RuntimeError(f"reference GPU kernels: {self.lib.refgpu_error().decode()}")

    @staticmethod
    def _p(t):
        return ct.c_void_p(t.data_ptr())

    def slice(self, dt, profile, cut_left, cut_right):
        profile.zero_()
        self._check(self.lib.refgpu_slice(self._p(dt), self._p(profile), cut_left,
                                          cut_right, profile.numel(), dt.numel(),
                                          self._stream()))

    @staticmethod
    def _stream():
        return ct.c_void_p(torch.cuda.current_stream().cuda_stream)

    @staticmethod
    def programme(prog):
        """Device copies of a programme (oracle/ref_cpu.programme): RF
        arrays as (n_turns+1, n_rf), acceleration kicks and drift tuples."""
        dev = "cuda"
        return dict(V=torch.tensor(prog["V"].T.copy(), device=dev),
                    om=torch.tensor(prog["om"].T.copy(), device=dev),
                    ph=torch.tensor(prog["ph"].T.copy(), device=dev),
                    acc=[float(x) for x in prog["acc"]], drift=prog["drift"])

    def setup(self, prog, n_turns_total):
        """Make `prog` the programme turn() uses by default."""
        self.prog = self.programme(prog)

    def turn(self, t, dt, dE, profile, cuts, bc, Z, n_fft, charge, ratio, factor, prog=None):
        n, S = dt.numel(), profile.numel()
        s = self._stream()
        p = prog or self.prog
        if Z is not None:
            spec = torch.fft.rfft(profile, n_fft)
            v = -(charge * E_CHARGE * ratio) * torch.fft.irfft(Z * spec, n_fft)
            v = v[:S].contiguous()
            self._check(self.lib.refgpu_lik(self._p(dt), self._p(dE), self._p(v),
                                            self._p(bc), charge, S, n, 0.0,
                                            self._p(factor), s))
        self._check(self.lib.refgpu_kick(self._p(dt), self._p(dE), p["V"].shape[1], charge,
                                         self._p(p["V"][t]), self._p(p["om"][t]),
                                         self._p(p["ph"][t]), n, p["acc"][t], s))
        a = p["drift"][t + 1]
        self._check(self.lib.refgpu_drift(self._p(dt), self._p(dE), 0, *[float(x) for x in a],
                                          n, s))
        self.slice(dt, profile, *cuts)
