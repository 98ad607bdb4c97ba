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
        self._stats_host = dict.fromkeys(_STAT_NAMES, 0.0)
        self._stats_dev = None      # device results of the last statistics()
        self._stats_pending = False
        self._stats_work = None     # scratch and ticket of the reduction
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
        """Mean and rms of the alive particles (beam.py:430-458) by one
        device reduction (blond_beam_statistics); nothing waits for it:
        mean_dt, sigma_dt, mean_dE, sigma_dE, epsn_rms_l are read back when
        first used.  stats_tensor() gives the device results."""
        if self._stats_work is None:
            self._stats_dev = torch.full((8,), float("nan"), dtype=torch.float64,
                                         device=self.dt.device)
            self._stats_work = (torch.empty(bm.STATS_SCRATCH, dtype=torch.float64,
                                            device=self.dt.device),
                                torch.zeros(1, dtype=torch.int32, device=self.dt.device))
        dt, dE = self.dt, self.dE
        if dE.dtype != dt.dtype:
            dE = dE.to(dt.dtype)
        bm.beam_statistics(dt, dE, self._id, out=self._stats_dev,
                           scratch=self._stats_work[0], ticket=self._stats_work[1])
        self._stats_pending = True

    def stats_tensor(self):
        """The device results of the last statistics(): [n_alive, mean_dt,
        sigma_dt, mean_dE, sigma_dE, epsn_rms_l, sum dt^2, sum dE^2]."""
        return self._stats_dev

    def _stat(self, name):
        if self._stats_pending:
            v = self._stats_dev.cpu().numpy()
            for k, x in zip(_STAT_NAMES, v[1:]):
                self._stats_host[k] = float(x)
            self._stats_pending = False
        return self._stats_host[name]

    def _set_stat(self, name, value):
        self._stat(name)  # settle pending device results first
        self._stats_host[name] = value


# attribute names Beam.statistics sets (beam.py:444-458), in the order of
# the device results after n_alive
_STAT_NAMES = ("mean_dt", "sigma_dt", "mean_dE", "sigma_dE", "epsn_rms_l",
               "_mpi_sumsq_dt", "_mpi_sumsq_dE")
for _name in _STAT_NAMES:
    setattr(Beam, _name, property(lambda self, n=_name: self._stat(n),
                                  lambda self, v, n=_name: self._set_stat(n, v)))
