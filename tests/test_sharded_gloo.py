"""One beam split over two ranks (torch.distributed gloo, CPU only).

The engine's sharded turn loop (blond_b200.engine.start_sharded /
run_sharded_turns: head, particle pass, histogram all-reduce) is driven
with the oracle's kernels on each rank's half of the bunch.  Because the
summed integer histogram equals the whole bunch's histogram, every particle
must come out bit-identical to the single-process oracle run -- the
property that makes the GPU path shard with one collective per turn.
"""
import datetime
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

N, S, TURNS = 4000, 256, 6


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _machine():
    from blond_b200.beam.beam import Proton
    from blond_b200.input_parameters.rf_parameters import RFStation
    from blond_b200.input_parameters.ring import Ring
    ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), TURNS)
    rf = RFStation(ring, [4620], [4.5e6], [0.0])
    return ring, rf


def _problem():
    import cpu_oracle as o
    from blond_b200.beam.distributions import _get_dE_from_dt, bigaussian_arrays
    ring, rf = _machine()
    centre = (rf.phi_s[0] - rf.phi_rf[0, 0]) / rf.omega_rf[0, 0]
    dt, dE = bigaussian_arrays(N, 0.4e-9, _get_dE_from_dt(ring, rf, 0.4e-9), centre, 11)
    cl, cr = centre - 1.25e-9, centre + 1.25e-9
    edges = np.linspace(cl, cr, S + 1)
    bc = (edges[:-1] + edges[1:]) / 2
    freq = np.fft.rfftfreq(S, (cr - cl) / S)
    Z = o.fast_resonator([5e6], [1.0], freq, [1e9]) / ((cr - cl) / S)
    return ring, rf, dt, dE, (cl, cr), bc, Z


def _worker(rank, world, port, out_path, fail_rank):
    sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]
    import cpu_oracle as o
    from blond_b200.engine import run_sharded_turns, start_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=30))
    try:
        ring, rf, dt_all, dE_all, cuts, bc, Z = _problem()
        lo, hi = rank * N // world, (rank + 1) * N // world
        dt, dE = dt_all[lo:hi].copy(), dE_all[lo:hi].copy()
        ratio = 1e10 / N  # the whole beam's charge per macro-particle
        st = {"turn": 0, "hist": torch.zeros(S, dtype=torch.int64), "v": None}

        def slice_local():
            st["hist"] = torch.from_numpy(o.histogram(dt, *cuts, S).astype(np.int64))

        def reduce():
            if rank == fail_rank and st["turn"] == 2:
                raise RuntimeError("injected failure on the host")
            dist.all_reduce(st["hist"], op=dist.ReduceOp.SUM)

        def refresh():
            st["profile"] = st["hist"].numpy().astype(np.float64)

        def head():
            refresh()
            st["v"] = o.induced_voltage(st["profile"], Z, S, 1.0, ratio, S)

        def particles():
            t = st["turn"]
            o.linear_interp_kick(dt, dE, st["v"], bc, 1.0, 0.0)
            o.kick(dt, dE, rf.voltage[:, t], rf.omega_rf[:, t], rf.phi_rf[:, t], 1.0,
                   -rf.delta_E[t])
            o.drift(dt, dE, 0, rf.t_rev[t + 1], rf.length_ratio, rf.alpha_order,
                    rf.eta_0[t + 1], rf.eta_1[t + 1], rf.eta_2[t + 1], rf.alpha_0[t + 1],
                    rf.alpha_1[t + 1], rf.alpha_2[t + 1], rf.beta[t + 1], rf.energy[t + 1])
            slice_local()
            st["turn"] += 1

        start_sharded(slice_local, reduce, refresh)
        run_sharded_turns(TURNS, head, particles, reduce, refresh)
        parts = [torch.zeros(N // world, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(parts, torch.from_numpy(dt))
        parts_e = [torch.zeros(N // world, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(parts_e, torch.from_numpy(dE))
        if rank == 0:
            np.savez(out_path, dt=torch.cat(parts).numpy(), dE=torch.cat(parts_e).numpy(),
                     profile=st["profile"])
    finally:
        dist.destroy_process_group()


def test_two_ranks_match_single_process(tmp_path):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cpu_oracle as o
    out = str(tmp_path / "sharded.npz")
    mp.spawn(_worker, args=(2, _free_port(), out, -1), nprocs=2, join=True)
    ring, rf, dt, dE, cuts, bc, Z = _problem()
    odt, odE, oprof, _ = o.track_oracle(dt, dE, ring, rf, cuts, bc, S, TURNS,
                                        impedance=(S, Z), intensity=1e10)
    got = np.load(out)
    np.testing.assert_array_equal(got["dt"], odt)
    np.testing.assert_array_equal(got["dE"], odE)
    np.testing.assert_array_equal(got["profile"], oprof[-1])


def test_a_rank_failing_on_the_host_ends_the_job(tmp_path):
    """Rank 1 raises before its third all-reduce; rank 0 must not wait
    forever: its collective ends with an error (peer gone / timeout) and the
    spawn reports the failure."""
    out = str(tmp_path / "never.npz")
    with pytest.raises(Exception):
        mp.spawn(_worker, args=(2, _free_port(), out, 1), nprocs=2, join=True)
    assert not os.path.exists(out)
