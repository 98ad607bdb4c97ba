"""Beam and particle types (blond/beam/beam.py:40-280, 430-458).

The macro-particle coordinates dt [s] and dE [eV] are structure-of-arrays
torch tensors on the current CUDA device, float64 for the 'double'
precision and float32 for 'single' (blond_b200.bmath.precision).
"""
from __future__ import annotations

import numpy as np
import torch
from scipy.constants import c, e, m_e, m_p

from .. import bmath as bm


class Particle:
    """Rest mass [eV] and charge [e] (beam.py:40-113)."""

    def __init__(self, user_mass: float, user_charge: float,
                 user_decay_rate: float = 0):
        if user_mass <= 0:
            raise RuntimeError("particle mass must be positive")
        self.mass = float(user_mass)
        self.charge = float(user_charge)
        self.decay_rate = float(user_decay_rate)


class Proton(Particle):
    def __init__(self):
        Particle.__init__(self, m_p * c**2 / e, 1)


class Electron(Particle):
    def __init__(self):
        Particle.__init__(self, m_e * c**2 / e, -1)


class Positron(Particle):
    def __init__(self):
        Particle.__init__(self, m_e * c**2 / e, 1)


def _to_device(x, dtype) -> torch.Tensor:
    dev = torch.device("cuda", torch.cuda.current_device())
    if isinstance(x, torch.Tensor):
        return x.to(device=dev, dtype=dtype).contiguous()
    return torch.from_numpy(np.ascontiguousarray(x)).to(device=dev, dtype=dtype)


class Beam:
    def __init__(self, ring, n_macroparticles: int, intensity: float, dt=None,
                 dE=None, dtype: torch.dtype | None = None):
        self.particle = ring.particle
        self.beta = float(ring.beta[0][0])
        self.gamma = float(ring.gamma[0][0])
        self.energy = float(ring.energy[0][0])
        self.momentum = float(ring.momentum[0][0])
        self.n_macroparticles = int(n_macroparticles)
        self.intensity = float(intensity)
        self.ratio = self.intensity / self.n_macroparticles
        dtype = dtype or bm.precision.torch_t
        n = self.n_macroparticles
        if dt is None:
            self.dt = torch.zeros(n, dtype=dtype, device="cuda")
        else:
            assert n == len(dt)
            self.dt = _to_device(dt, dtype)
        if dE is None:
            self.dE = torch.zeros(n, dtype=dtype, device="cuda")
        else:
            assert n == len(dE)
            self.dE = _to_device(dE, dtype)
        self.mean_dt = self.mean_dE = 0.0
        self.sigma_dt = self.sigma_dE = 0.0
        self.epsn_rms_l = 0.0
        self.n_macroparticles_eliminated = 0
        self._id = None

    @property
    def id(self) -> torch.Tensor:
        """Particle ids (1..N; 0 marks a lost particle), allocated on use."""
        if self._id is None:
            self._id = torch.arange(1, self.n_macroparticles + 1,
                                    dtype=torch.int64, device=self.dt.device)
        return self._id

    @id.setter
    def id(self, v):
        self._id = _to_device(v, torch.int64)

    @property
    def n_macroparticles_alive(self) -> int:
        if self._id is None:
            return self.n_macroparticles
        return int(torch.count_nonzero(self._id))

    def statistics(self):
        """Mean and rms of the alive particles (beam.py:430-458)."""
        if self._id is None:
            dt, dE = self.dt.double(), self.dE.double()
        else:
            alive = self._id != 0
            dt, dE = self.dt[alive].double(), self.dE[alive].double()
        self.mean_dt = float(dt.mean())
        self.sigma_dt = float(dt.std(unbiased=False))
        self.mean_dE = float(dE.mean())
        self.sigma_dE = float(dE.std(unbiased=False))
        self.epsn_rms_l = float(np.pi * self.sigma_dE * self.sigma_dt)
