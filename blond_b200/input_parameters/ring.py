"""Ring: per-turn synchronous programme (blond/input_parameters/ring.py:217-462).

Host-side parameter source for the tracker.  Supports one section with a
momentum (or total/kinetic energy) given as a scalar or as a per-turn array
of n_turns+1 values, and momentum compaction factors alpha_0..2 (scalar or
per-turn).  Arrays have the reference's [n_sections, n_turns+1] shape.
"""
from __future__ import annotations

import numpy as np
from scipy.constants import c


def _per_turn(x, n_turns: int, name: str) -> np.ndarray:
    a = np.asarray(x, dtype=float)
    if a.ndim == 0 or a.size == 1:
        return np.full((1, n_turns + 1), float(a.reshape(-1)[0]))
    a = a.reshape(-1)
    if a.size != n_turns + 1:
        raise NotImplementedError(
            f"{name}: give a scalar or one value per turn (n_turns+1 = "
            f"{n_turns + 1}); time-interpolated programmes are not supported")
    return a.reshape(1, -1).copy()


class Ring:
    def __init__(self, ring_length, alpha_0, synchronous_data, particle,
                 n_turns: int = 1, synchronous_data_type: str = "momentum",
                 bending_radius=None, n_sections: int = 1, alpha_1=None,
                 alpha_2=None, ring_options=None):
        if int(n_sections) != 1:
            raise NotImplementedError("only one RF section is supported")
        self.n_turns = int(n_turns)
        self.n_sections = 1
        self.ring_length = np.array(ring_length, ndmin=1, dtype=float)
        self.ring_circumference = float(np.sum(self.ring_length))
        self.ring_radius = self.ring_circumference / (2 * np.pi)
        self.bending_radius = bending_radius
        self.particle = particle
        data = _per_turn(synchronous_data, self.n_turns, "synchronous_data")
        mass = particle.mass
        if synchronous_data_type == "momentum":
            self.momentum = data
        elif synchronous_data_type == "total energy":
            self.momentum = np.sqrt(data**2 - mass**2)
        elif synchronous_data_type == "kinetic energy":
            self.momentum = np.sqrt((data + mass) ** 2 - mass**2)
        else:
            raise NotImplementedError(synchronous_data_type)
        # ring.py:297-317
        self.beta = np.sqrt(1 / (1 + (mass / self.momentum) ** 2))
        self.gamma = np.sqrt(1 + (self.momentum / mass) ** 2)
        self.energy = np.sqrt(self.momentum**2 + mass**2)
        self.kin_energy = np.sqrt(self.momentum**2 + mass**2) - mass
        self.t_rev = np.dot(self.ring_length, 1 / (self.beta * c))
        self.cycle_time = np.cumsum(self.t_rev)
        self.f_rev = 1 / self.t_rev
        self.omega_rev = 2 * np.pi * self.f_rev
        self.delta_E = np.diff(self.energy, axis=1)
        self.alpha_0 = _per_turn(alpha_0, self.n_turns, "alpha_0")
        self.alpha_order = 0
        if alpha_1 is not None:
            self.alpha_1 = _per_turn(alpha_1, self.n_turns, "alpha_1")
            self.alpha_order = 1
        else:
            self.alpha_1 = np.zeros(self.alpha_0.shape)
        if alpha_2 is not None:
            self.alpha_2 = _per_turn(alpha_2, self.n_turns, "alpha_2")
            self.alpha_order = 2
        else:
            self.alpha_2 = np.zeros(self.alpha_0.shape)
        self.eta_generation()

    def eta_generation(self):
        """Slippage factors eta_0..2 (ring.py:380-462)."""
        b, g = self.beta[0], self.gamma[0]
        a0, a1, a2 = self.alpha_0[0], self.alpha_1[0], self.alpha_2[0]
        z = np.zeros((1, self.n_turns + 1))
        self.eta_0 = (a0 - g ** (-2.0)).reshape(1, -1)
        self.eta_1 = z.copy()
        self.eta_2 = z.copy()
        if self.alpha_order >= 1:
            self.eta_1 = (3 * b**2 / (2 * g**2) + a1 - a0 * self.eta_0[0]).reshape(1, -1)
        if self.alpha_order >= 2:
            self.eta_2 = (-(b**2) * (5 * b**2 - 1) / (2 * g**2) + a2 - 2 * a0 * a1
                          + a1 / g**2 + a0**2 * self.eta_0[0]
                          - 3 * b**2 * a0 / (2 * g**2)).reshape(1, -1)
