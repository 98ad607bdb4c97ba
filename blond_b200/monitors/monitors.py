"""BunchMonitor and SlicesMonitor (blond/monitors/monitors.py:36-508).

The reference computes Beam.statistics() on the host every turn and keeps a
host buffer it flushes to an HDF5 file every `buffer_time` turns.  Here the
statistics are one device reduction per turn (blond_beam_statistics) whose
8 results are copied, on the device, into row i of a device buffer; the
host sees the buffer only when it is flushed, so a turn costs no host
synchronisation.  The per-turn values of a BeamFeedback and a profile fit,
which live on the host, go to host buffers as in the reference.

Files: with h5py importable, `filename + '.h5'` with the reference's group
('Beam' / 'Slices'), dataset names, shapes and dtypes.  Without it (this
package does not require h5py), the same datasets are written with
numpy.savez to `filename + '.npz'`.
"""
from __future__ import annotations

import os

import numpy as np
import torch

try:  # optional: the reference's file format
    import h5py as _h5py
except ImportError:  # pragma: no cover - depends on the environment
    _h5py = None

# stats_tensor() index of each BunchMonitor statistic
_STATS = (("n_macroparticles_alive", 0), ("mean_dt", 1), ("mean_dE", 3),
          ("sigma_dt", 2), ("sigma_dE", 4), ("epsn_rms_l", 5))
_LOOP = ("PL_omegaRF", "PL_phiRF", "PL_bunch_phase", "PL_phase_corr", "PL_omegaRF_corr",
         "SL_dphiRF", "RL_drho")


def _makedirs_for(filename):
    dirname = os.path.dirname(filename)
    if dirname:
        os.makedirs(dirname, exist_ok=True)


def _save(filename, group, data):
    """Write the datasets of one group: HDF5 if h5py is there, else .npz."""
    if _h5py is not None:
        with _h5py.File(filename + ".h5", "w") as f:
            g = f.require_group(group)
            for k, v in data.items():
                g.create_dataset(k, data=v)
    else:
        np.savez(filename + ".npz", **data)


class BunchMonitor:
    """Bunch statistics every turn, flushed to file every buffer_time turns
    (monitors.py:36-466).  Phase noise feedback is not supported."""

    def __init__(self, ring, rf_parameters, beam, filename, buffer_time=None, profile=None,
                 phase_loop=None, lhc_noise_feedback=None):
        if lhc_noise_feedback is not None:
            raise NotImplementedError("LHCNoiseFB is not supported")
        self.filename = str(filename)
        self.n_turns = ring.n_turns
        self.i_turn = 0
        self.buffer_time = buffer_time if buffer_time is not None else self.n_turns
        self.rf_params = rf_parameters
        self.beam = beam
        self.profile = profile
        self.fit_option = profile is not None and profile.fit_option is not None
        self.phase_loop = phase_loop
        self.lhc_noise_feedback = None
        self.init_data(self.filename, (self.n_turns + 1,))
        self.track()

    def init_data(self, filename, dims):
        """monitors.py:140-325: the datasets, with the state at turn 0."""
        self.beam.statistics()
        _makedirs_for(filename)
        self.data = {name: np.zeros(dims, dtype=np.float32) for name, _ in _STATS}
        st = self.beam.stats_tensor().cpu().numpy()
        for name, k in _STATS:
            self.data[name][0] = st[k]
        if self.fit_option:
            self.data["bunch_length"] = np.zeros(dims, dtype=np.float32)
            self.data["bunch_length"][0] = self.profile.bunchLength
        if self.phase_loop is not None:
            for name in _LOOP:
                self.data[name] = np.zeros(dims, dtype=np.float64 if name == "PL_omegaRF"
                                           else np.float32)
            self._loop_values(self.data, 0)
        self._write()
        self.init_buffer()

    def _loop_values(self, dst, i):
        rf, pl = self.rf_params, self.phase_loop
        dst["PL_omegaRF"][i] = rf.omega_rf[0, self.i_turn]
        dst["PL_phiRF"][i] = rf.phi_rf[0, self.i_turn]
        dst["PL_bunch_phase"][i] = pl.phi_beam
        dst["PL_phase_corr"][i] = pl.dphi
        dst["PL_omegaRF_corr"][i] = pl.domega_rf
        dst["SL_dphiRF"][i] = rf.dphi_rf[0]
        dst["RL_drho"][i] = pl.drho

    def init_buffer(self):
        """monitors.py:327-356: the statistics buffer lives on the device."""
        self.b_stats = torch.zeros((self.buffer_time, 8), dtype=torch.float64,
                                   device=self.beam.dt.device)
        self.b_host = {}
        if self.fit_option:
            self.b_host["bunch_length"] = np.zeros(self.buffer_time)
        if self.phase_loop is not None:
            for name in _LOOP:
                self.b_host[name] = np.zeros(self.buffer_time)

    def write_buffer(self):
        """monitors.py:358-386: row i_turn % buffer_time, copied on the
        device."""
        i = self.i_turn % self.buffer_time
        self.b_stats[i].copy_(self.beam.stats_tensor())
        if self.fit_option:
            self.b_host["bunch_length"][i] = self.profile.bunchLength
        if self.phase_loop is not None:
            self._loop_values(self.b_host, i)

    def track(self):
        """monitors.py:125-138."""
        self.beam.statistics()
        self.write_buffer()
        self.i_turn += 1
        if self.i_turn > 0 and (self.i_turn % self.buffer_time) == 0:
            self.write_data()
            self.init_buffer()

    def write_data(self):
        """monitors.py:388-455: the buffered turns into their rows."""
        i1, i2 = self.i_turn - self.buffer_time, self.i_turn
        st = self.b_stats.cpu().numpy()
        for name, k in _STATS:
            self.data[name][i1:i2] = st[:, k]
        for name, buf in self.b_host.items():
            self.data[name][i1:i2] = buf
        self._write()

    def _write(self):
        _save(self.filename, "Beam", self.data)

    def open(self):
        pass

    def close(self):
        pass


class SlicesMonitor:
    """The profile of every turn (monitors.py:470-508): one column per turn
    of an (n_slices, n_turns) dataset 'n_macroparticles'.  Columns gather in
    a device buffer of `buffer_size` turns and move to the host when it is
    full; close() writes the file."""

    def __init__(self, filename, n_turns, profile, buffer_size: int = 128):
        _makedirs_for(str(filename))
        self.filename = str(filename)
        self.n_turns = int(n_turns)
        self.i_turn = 0
        self.profile = profile
        self.buffer_size = int(buffer_size)
        S = int(profile.n_slices)
        self.n_macroparticles = np.zeros((S, self.n_turns), dtype=np.float32)
        self._buf = torch.zeros((self.buffer_size, S), dtype=torch.float32,
                                device=profile.n_macroparticles.device)
        self._first = 0

    def track(self):
        if self.i_turn >= self.n_turns:
            raise IndexError("SlicesMonitor: more turns than n_turns")
        self._buf[self.i_turn - self._first].copy_(self.profile.n_macroparticles)
        self.i_turn += 1
        if self.i_turn - self._first == self.buffer_size:
            self._drain()

    def _drain(self):
        m = self.i_turn - self._first
        if m:
            self.n_macroparticles[:, self._first:self.i_turn] = self._buf[:m].cpu().numpy().T
        self._first = self.i_turn

    def close(self):
        self._drain()
        _save(self.filename, "Slices", {"n_macroparticles": self.n_macroparticles})
