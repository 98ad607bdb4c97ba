"""Differentiable N-turn tracking with a hand-written adjoint.

``AdjointTracker(...)(dt0, dE0, voltage, phi, impedance)`` runs the
per-turn map of the reference main loop -- induced voltage of the
turn-start profile and its interpolated kick
(blond/impedances/impedance.py:113-146), RF kick and simple drift
(blond/trackers/tracker.py:521-615) -- for ``n_turns`` turns and returns the
final coordinates and profile as outputs of a ``torch.autograd.Function``.
Any torch loss of those outputs back-propagates through the adjoint kernels
(blond_b200/csrc/adjoint.cu) to

* the per-turn RF voltage and phase programmes ``voltage[t, j]``,
  ``phi[t, j]``,
* the impedance (complex, n_fft/2+1 values) -- and through
  ``resonator_impedance`` to the resonators' R_s, f_r and Q,
* the initial coordinates.

The profile is a cloud-in-cell deposit on the bin centres, which is
continuous in every dt; the reference's smooth_histogram
(blond/cpp_routines/histogram.cpp:75-132) moves a whole macro-particle by
two bins where it crosses a bin centre, so it has no useful derivative.

Memory: the forward keeps dt/dE every ``checkpoint_every`` turns plus the
induced voltage and profile spectrum of every turn; the backward recomputes
one segment at a time from its checkpoint (bit-identical: the stored
voltages are reused) holding that segment's dt, then runs its turns
backwards.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import torch
from scipy.constants import e as E_CHARGE

from . import _lib

PREC = {"f64": 0, "f32p64": 1}


def _p(t: torch.Tensor | None) -> ct.c_void_p:
    return ct.c_void_p(t.data_ptr() if t is not None else 0)


def _stream() -> ct.c_void_p:
    return ct.c_void_p(torch.cuda.current_stream().cuda_stream)


def resonator_impedance(R_S, frequency_R, Q, n_fft: int, bin_size: float) -> torch.Tensor:
    """Z[k] = sum_r R_r / (1 + j Q_r (f_k/f_r - f_r/f_k)) / bin_size on
    f = rfftfreq(n_fft, bin_size), Z[0] = 0 -- Resonators.imped_calc
    (impedance_sources.py:382-414, fast_resonator.cpp:19-74) summed and
    scaled as InducedVoltageFreq.sum_impedances (impedance.py:846-890) --
    written with differentiable torch operations (complex128)."""
    R = torch.as_tensor(R_S, dtype=torch.float64).reshape(-1)
    fr = torch.as_tensor(frequency_R, dtype=torch.float64).reshape(-1)
    q = torch.as_tensor(Q, dtype=torch.float64).reshape(-1)
    dev = R.device
    f = torch.arange(1, n_fft // 2 + 1, dtype=torch.float64, device=dev) / (n_fft * bin_size)
    x = f[None, :] / fr[:, None] - fr[:, None] / f[None, :]
    z = R[:, None] / torch.complex(torch.ones_like(x), q[:, None] * x)
    z = z.sum(dim=0) / bin_size
    return torch.cat([torch.zeros(1, dtype=torch.complex128, device=dev), z])


class AdjointTracker:
    """The differentiable map of ``n_turns`` turns starting at
    ``rf_station.counter[0]``.

    ring, rf_station: the drop-in objects (drift and RF frequency
    programmes; the voltage and phase programmes are inputs of the call).
    n_macroparticles, intensity: give the charge per macro-particle of the
    induced voltage (ratio = intensity / n_macroparticles, beam.py:266).
    cut_left, cut_right, n_slices: the profile window (Profile's bin
    centres).  n_fft: FFT length of the impedance (default n_slices).
    precision: "f32p64" (float dE, FP64 RF phase and drift) or "f64".
    """

    def __init__(self, ring, rf_station, n_macroparticles: int, intensity: float,
                 cut_left: float, cut_right: float, n_slices: int, n_turns: int,
                 n_fft: int | None = None, precision: str = "f32p64",
                 checkpoint_every: int = 50):
        if precision not in PREC:
            raise ValueError(f"precision must be one of {list(PREC)}")
        rf = rf_station
        if rf.n_rf > 4:
            raise NotImplementedError("the adjoint kernels take at most 4 RF systems")
        self.precision = precision
        self.n = int(n_macroparticles)
        self.S = int(n_slices)
        self.n_fft = int(n_fft or n_slices)
        if self.n_fft < self.S or self.n_fft % 2:
            raise ValueError("n_fft must be even and >= n_slices")
        self.T = int(n_turns)
        self.K = max(1, int(checkpoint_every))
        t0 = int(rf.counter[0])
        if t0 + self.T > rf.n_turns:
            raise ValueError("n_turns runs past the RF programme")
        self.t0 = t0
        self.n_rf = int(rf.n_rf)
        self.charge = float(rf.particle.charge)
        self.cut_left, self.cut_right = float(cut_left), float(cut_right)
        self.bin_size = (self.cut_right - self.cut_left) / self.S
        self.bc0 = self.cut_left + 0.5 * self.bin_size
        self.inv_w = self.S / (self.cut_right - self.cut_left)
        self.scale = self.charge * E_CHARGE * float(intensity) / self.n
        dev = torch.device("cuda")
        sl = slice(t0, t0 + self.T)
        om = np.asarray(rf.omega_rf, dtype=np.float64)[:, sl].T
        self.omega = torch.tensor(np.ascontiguousarray(om), device=dev)
        self.acc = (-np.asarray(rf.delta_E, dtype=np.float64)[sl]).tolist()
        nx = slice(t0 + 1, t0 + self.T + 1)
        self.drift_c = (np.asarray(rf.t_rev, float)[nx] * float(rf.length_ratio)
                        * np.asarray(rf.eta_0, float)[nx]
                        / (np.asarray(rf.beta, float)[nx] ** 2
                           * np.asarray(rf.energy, float)[nx])).tolist()
        # host copies for the C turn loops
        self._acc_h = (ct.c_double * self.T)(*self.acc)
        self._drift_h = (ct.c_double * self.T)(*self.drift_c)
        _lib.load()

    # ------------------------------------------------------------ helpers
    def impedance(self, R_S, frequency_R, Q) -> torch.Tensor:
        """Resonator impedance on this tracker's FFT grid (differentiable)."""
        return resonator_impedance(R_S, frequency_R, Q, self.n_fft, self.bin_size)

    def bin_centers(self) -> torch.Tensor:
        return self.bc0 + torch.arange(self.S, dtype=torch.float64, device="cuda") / self.inv_w

    def profile(self, dt: torch.Tensor) -> torch.Tensor:
        """Cloud-in-cell profile of dt (no gradient)."""
        out = torch.zeros(self.S, dtype=torch.float64, device="cuda")
        dt = dt.detach().to(torch.float64).contiguous()
        _lib.call("blond_adjoint_deposit", _p(dt), dt.numel(), self.S, self.bc0,
                  self.inv_w, _p(out), _stream())
        return out

    def __call__(self, dt0, dE0, voltage, phi, impedance=None):
        """Track n_turns turns.  voltage, phi: (n_turns, n_rf) float64 CUDA
        tensors; impedance: complex128 (n_fft/2+1) or None.  Returns
        (dt, dE, profile) after the last turn."""
        return _AdjointMap.apply(self, dt0, dE0, voltage, phi, impedance)

    # ------------------------------------------------------------ kernels
    def _forward_turn(self, t, dt_in, dE_in, dt_out, dE_out, voltage, phi, vind, prof_out):
        _lib.call("blond_adjoint_forward_turn", PREC[self.precision], _p(dt_in), _p(dE_in),
                  _p(dt_out), _p(dE_out), self.n, self.n_rf, _p(voltage[t]),
                  _p(self.omega[t]), _p(phi[t]), self.acc[t], self.charge,
                  self.drift_c[t], _p(vind), self.S, self.bc0, self.inv_w, _p(prof_out),
                  _stream())

    def _spectral(self, mode, x, H, y, spec, accum=None):
        _lib.call("blond_adjoint_spectral", mode, _p(x), self.S, _p(H), self.n_fft,
                  self.scale, _p(y), _p(spec), _p(accum), _stream())


def _real_view(z: torch.Tensor) -> torch.Tensor:
    return torch.view_as_real(z.contiguous())


class _AdjointMap(torch.autograd.Function):
    @staticmethod
    def forward(ctx, tr: AdjointTracker, dt0, dE0, voltage, phi, Z):
        dev = torch.device("cuda")
        edt = torch.float64 if tr.precision == "f64" else torch.float32
        if dt0.numel() != tr.n or dE0.numel() != tr.n:
            raise ValueError(f"expected {tr.n} particles")
        if tuple(voltage.shape) != (tr.T, tr.n_rf) or tuple(phi.shape) != (tr.T, tr.n_rf):
            raise ValueError(f"voltage and phi must be ({tr.T}, {tr.n_rf})")
        V = voltage.detach().to(dev, torch.float64).contiguous()
        P = phi.detach().to(dev, torch.float64).contiguous()
        dt = dt0.detach().to(dev, torch.float64).clone().contiguous()
        dE = dE0.detach().to(dev, edt).clone().contiguous()
        has_z = Z is not None
        M1 = tr.n_fft // 2 + 1
        Zd = Z.detach().to(dev, torch.complex128).contiguous() if has_z else None
        if has_z and Zd.numel() != M1:
            raise ValueError(f"impedance must have n_fft/2+1 = {M1} values")
        vind = torch.empty(tr.T, tr.S, dtype=torch.float64, device=dev) if has_z else None
        spec = torch.empty(tr.T, M1, dtype=torch.complex128, device=dev) if has_z else None
        prof = torch.zeros(tr.T + 1, tr.S, dtype=torch.float64, device=dev)
        nseg = (tr.T + tr.K - 1) // tr.K
        ckpt_dt = torch.empty(nseg, tr.n, dtype=torch.float64, device=dev)
        ckpt_dE = torch.empty(nseg, tr.n, dtype=edt, device=dev)
        Zr = _real_view(Zd) if has_z else None
        # the turn loop runs in C (blond_adjoint_forward_run): the turn-0
        # profile, then per turn checkpoints, induced voltage and spectrum,
        # forward turn and profile
        _lib.call("blond_adjoint_forward_run", PREC[tr.precision], _p(dt), _p(dE), tr.n,
                  tr.n_rf, tr.T, _p(V), _p(tr.omega), _p(P),
                  ct.cast(tr._acc_h, ct.c_void_p), ct.cast(tr._drift_h, ct.c_void_p),
                  tr.charge, _p(Zr), tr.n_fft, tr.scale, _p(vind),
                  _p(_real_view(spec) if has_z else None), _p(prof), tr.S, tr.bc0, tr.inv_w,
                  tr.K, _p(ckpt_dt), _p(ckpt_dE), _stream())
        ckpt = (ckpt_dt, ckpt_dE)
        ctx.tr = tr
        ctx.saved = (V, P, Zd, vind, spec, ckpt)
        ctx.edt = (dt0.dtype, dE0.dtype)
        out_prof = prof[tr.T].clone()
        del prof
        return dt, dE, out_prof

    @staticmethod
    def backward(ctx, g_dt, g_dE, g_prof):
        tr = ctx.tr
        V, P, Zd, vind, spec, ckpt = ctx.saved
        dev = V.device
        n, S, T, K = tr.n, tr.S, tr.T, tr.K
        has_z = Zd is not None
        lam_dt = (g_dt.detach().to(torch.float64).clone().contiguous() if g_dt is not None
                  else torch.zeros(n, dtype=torch.float64, device=dev))
        lam_dE = (g_dE.detach().to(torch.float64).clone().contiguous() if g_dE is not None
                  else torch.zeros(n, dtype=torch.float64, device=dev))
        lam_p = g_prof.detach().to(torch.float64).contiguous() if g_prof is not None else None
        grad_rf = torch.zeros(T, 2 * tr.n_rf, dtype=torch.float64, device=dev)
        M1 = tr.n_fft // 2 + 1
        G = torch.zeros(M1, dtype=torch.complex128, device=dev) if has_z else None
        Zc = _real_view(Zd.conj().resolve_conj()) if has_z else None
        lam_v = torch.zeros(T, S, dtype=torch.float64, device=dev) if has_z else None
        lam_pt = torch.empty(T, S, dtype=torch.float64, device=dev) if has_z else None
        states = torch.empty(K + 1, n, dtype=torch.float64, device=dev)
        ckpt_dt, ckpt_dE = ckpt
        dE_work = torch.empty_like(ckpt_dE[0])
        # the backward sweep runs in C (blond_adjoint_backward_run): per
        # segment the recomputed turn-start coordinates, then the backward
        # turns and the transposed induced-voltage transform, last the
        # deposit adjoint of the turn-0 profile
        _lib.call("blond_adjoint_backward_run", PREC[tr.precision], n, tr.n_rf, T, _p(V),
                  _p(tr.omega), _p(P), ct.cast(tr._acc_h, ct.c_void_p),
                  ct.cast(tr._drift_h, ct.c_void_p), tr.charge, _p(Zc), tr.n_fft, tr.scale,
                  _p(vind), _p(_real_view(spec) if has_z else None), S, tr.bc0, tr.inv_w, K,
                  _p(ckpt_dt), _p(ckpt_dE), _p(states), _p(dE_work), _p(lam_dt), _p(lam_dE),
                  _p(lam_p), _p(lam_v), _p(lam_pt), _p(grad_rf),
                  _p(_real_view(G) if has_z else None), _stream())
        grad_V = grad_rf[:, :tr.n_rf].contiguous()
        grad_phi = grad_rf[:, tr.n_rf:].contiguous()
        grad_Z = None
        if has_z:
            # dL = -(scale / n_fft) sum_k w_k Re(dZ_k G_k), w = 1 at DC and
            # Nyquist, 2 elsewhere; torch's complex gradient is conj(dL/dZ)
            w = torch.full((M1,), 2.0, dtype=torch.float64, device=dev)
            w[0] = 1.0
            w[-1] = 1.0
            grad_Z = (-(tr.scale / tr.n_fft) * w) * G.conj()
        dt_dtype, dE_dtype = ctx.edt
        return (None, lam_dt.to(dt_dtype), lam_dE.to(dE_dtype), grad_V, grad_phi, grad_Z)


def bunch_loss(profile: torch.Tensor, target: torch.Tensor, bin_centers: torch.Tensor,
               time_unit: float = 1e-9) -> torch.Tensor:
    """RMS bunch length squared of the profile (time_unit^2) plus the L2
    mismatch of the profile normalised to sum 1 against target.

    The RMS length is the reference's line-density definition
    (blond/toolbox/filters_and_fitting.py:158-172: trapezoid moments of the
    normalised profile, bunch length = 4 sigma); particles outside the
    profile window do not enter, as in the reference."""
    w = torch.ones_like(profile)
    w[0] = 0.5
    w[-1] = 0.5
    wp = w * profile
    norm = wp.sum()
    mu = (wp * bin_centers).sum() / norm
    sig2 = (wp * (bin_centers - mu) ** 2).sum() / norm
    return sig2 / time_unit**2 + ((profile / profile.sum() - target) ** 2).sum()


def gaussian_target(n_slices: int, cut_left: float, cut_right: float, centre: float,
                    sigma: float) -> torch.Tensor:
    """A Gaussian on the bin centres, normalised to sum 1."""
    w = (cut_right - cut_left) / n_slices
    bc = cut_left + (torch.arange(n_slices, dtype=torch.float64) + 0.5) * w
    g = torch.exp(-0.5 * ((bc - centre) / sigma) ** 2)
    return (g / g.sum()).cuda()


__all__ = ["AdjointTracker", "resonator_impedance", "bunch_loss", "gaussian_target"]
