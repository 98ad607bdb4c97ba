"""The differentiable map on the GPU and its hand-written adjoint.

Bars: FP64 forward against the numpy restatement (oracle/adjoint_oracle.py)
within 1e-12 normwise; gradients against central finite differences of
that restatement (FP64, relative step 1e-6) within 1e-4 relative -- the
bar of the differentiable form; gradients independent of the checkpoint
interval to 1e-12; at the C4 size (2e6 particles, 1024 slices, 500 turns,
checkpoints every 50; broadband resonator 1 MOhm / 1 GHz / Q 1 at
intensity 3e9, a bunch that stays stable over the 500 turns) the FP64
adjoint against finite differences of the GPU FP64 forward within 1e-4,
and the F32P64 adjoint against the FP64 one over 100 turns.
"""
import numpy as np
import pytest
import torch

import adjoint_oracle as ao
from conftest import normwise
from blond_b200.adjoint import AdjointTracker, bunch_loss, gaussian_target
from blond_b200.beam.beam import Proton
from blond_b200.beam.distributions import _get_dE_from_dt, bigaussian_arrays
from blond_b200.impedances.impedance import InducedVoltageFreq
from blond_b200.impedances.impedance_sources import Resonators
from blond_b200.input_parameters.rf_parameters import RFStation
from blond_b200.input_parameters.ring import Ring

pytestmark = pytest.mark.gpu

RES = (np.array([5e6]), np.array([1e9]), np.array([1.0]))  # R_s, f_r, Q


def make(n, S, T, precision="f64", K=50, intensity=1e10, seed=3):
    ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), T)
    rf = RFStation(ring, [4620], [4.5e6], [0.0])
    centre = (rf.phi_s[0] - rf.phi_rf[0, 0]) / rf.omega_rf[0, 0]
    dt0, dE0 = bigaussian_arrays(n, 0.4e-9, _get_dE_from_dt(ring, rf, 0.4e-9), centre, seed)
    cl, cr = centre - 1.25e-9, centre + 1.25e-9
    tr = AdjointTracker(ring, rf, n, intensity, cl, cr, S, T, precision=precision,
                        checkpoint_every=K)
    target = gaussian_target(S, cl, cr, centre, 0.35e-9)
    return ring, rf, tr, dt0, dE0, target


def oracle_args(tr, V, phi, R, fr, Q):
    om = tr.omega.cpu().numpy()
    Z = ao.resonator_impedance(R, fr, Q, tr.n_fft, tr.bin_size) if R is not None else None
    return (V, om, phi, np.array(tr.acc), np.array(tr.drift_c), tr.charge, Z, tr.scale, tr.S,
            tr.n_fft, tr.bc0, tr.inv_w)


def oracle_loss(tr, dt0, dE0, V, phi, R, fr, Q, target):
    dt, _, p, _ = ao.track(dt0, dE0, *oracle_args(tr, V, phi, R, fr, Q))
    return ao.bunch_loss(p, target, tr.bin_centers().cpu().numpy())


def gpu_grads(tr, dt0, dE0, V, phi, R, fr, Q, target):
    dev = "cuda"
    Vt = torch.tensor(V, device=dev, requires_grad=True)
    Pt = torch.tensor(phi, device=dev, requires_grad=True)
    Rt, frt, Qt = (torch.tensor(x, device=dev, requires_grad=True) for x in (R, fr, Q))
    dtt = torch.tensor(dt0, device=dev, requires_grad=True)
    dEt = torch.tensor(dE0, device=dev, requires_grad=True)
    dt, dE, p = tr(dtt, dEt, Vt, Pt, tr.impedance(Rt, frt, Qt))
    L = bunch_loss(p, target, tr.bin_centers())
    L.backward()
    g = {k: v.grad.cpu().numpy() for k, v in
         dict(V=Vt, phi=Pt, R=Rt, fr=frt, Q=Qt, dt0=dtt, dE0=dEt).items()}
    return float(L), g, (dt, dE, p)


def test_resonator_impedance_matches_dropin(cuda):
    _, _, tr, dt0, dE0, _ = make(1000, 256, 2)
    from blond_b200.beam.beam import Beam
    from blond_b200.beam.profile import CutOptions, Profile
    ring = Ring(6911.5, 1 / 18**2, 26e9, Proton(), 2)
    beam = Beam(ring, 1000, 1e10, dt=dt0, dE=dE0)
    prof = Profile(beam, CutOptions(cut_left=tr.cut_left, cut_right=tr.cut_right,
                                    n_slices=256))
    iv = InducedVoltageFreq(beam, prof, [Resonators([5e6, 1e5], [1e9, 2e8], [1.0, 300.0])])
    z = tr.impedance(torch.tensor([5e6, 1e5]), torch.tensor([1e9, 2e8]),
                     torch.tensor([1.0, 300.0]))
    assert normwise(z.cpu().numpy(), iv.total_impedance.cpu().numpy()) < 1e-13


def test_forward_matches_oracle(cuda):
    n, S, T = 20000, 64, 30
    _, rf, tr, dt0, dE0, _ = make(n, S, T, intensity=1e10)
    V = np.full((T, 1), 4.5e6)
    phi = np.zeros((T, 1))
    dt, dE, p = tr(torch.tensor(dt0, device="cuda"), torch.tensor(dE0, device="cuda"),
                   torch.tensor(V, device="cuda"), torch.tensor(phi, device="cuda"),
                   tr.impedance(*RES))
    odt, odE, op, ov = ao.track(dt0, dE0, *oracle_args(tr, V, phi, *RES))
    assert normwise(dt.cpu().numpy(), odt) < 1e-12
    assert normwise(dE.cpu().numpy(), odE) < 1e-12
    assert normwise(p.cpu().numpy(), op) < 1e-12
    # the induced voltage matters in this case
    assert np.abs(ov[-1]).max() > 1e4


@pytest.mark.parametrize("K", [1, 7])
def test_gradients_match_finite_differences(cuda, K):
    n, S, T = 4000, 64, 20
    _, rf, tr, dt0, dE0, target = make(n, S, T, K=K, intensity=1e10)
    V = np.full((T, 1), 4.5e6) * (1 + 0.01 * np.sin(np.arange(T))[:, None])
    phi = 0.01 * np.cos(np.arange(T))[:, None]
    R, fr, Q = RES
    L, g, _ = gpu_grads(tr, dt0, dE0, V, phi, R, fr, Q, target)
    tg = target.cpu().numpy()
    assert abs(L - oracle_loss(tr, dt0, dE0, V, phi, R, fr, Q, tg)) < 1e-12 * abs(L)

    def fd(kind, idx, h):
        args = dict(V=V.copy(), phi=phi.copy(), R=R.copy(), fr=fr.copy(), Q=Q.copy(),
                    dt0=dt0.copy(), dE0=dE0.copy())
        up, dn = {k: v.copy() for k, v in args.items()}, {k: v.copy() for k, v in args.items()}
        up[kind][idx] += h
        dn[kind][idx] -= h
        f = lambda a: oracle_loss(tr, a["dt0"], a["dE0"], a["V"], a["phi"], a["R"],  # noqa
                                  a["fr"], a["Q"], tg)
        return (f(up) - f(dn)) / (2 * h)

    checks = [("V", (0, 0)), ("V", (T // 2, 0)), ("V", (T - 1, 0)), ("phi", (0, 0)),
              ("phi", (T - 2, 0)), ("R", 0), ("fr", 0), ("Q", 0), ("dt0", 17), ("dE0", 17)]
    for kind, idx in checks:
        x0 = {"V": V, "phi": phi, "R": R, "fr": fr, "Q": Q, "dt0": dt0, "dE0": dE0}[kind][idx]
        h = 1e-6 * abs(x0)
        if kind == "phi":
            h = 1e-6  # rad: a phase programme of 0.01 rad has no natural scale
        if kind == "dt0":
            h = 1e-6 * 0.4e-9
        ref = fd(kind, idx, h)
        got = g[kind][idx]
        assert abs(got - ref) <= 1e-4 * abs(ref), (kind, idx, got, ref)


def test_gradients_independent_of_checkpoint_interval(cuda):
    n, S, T = 20000, 128, 24
    out = []
    for K in (1, 5, 24):
        _, rf, tr, dt0, dE0, target = make(n, S, T, K=K, intensity=1e10)
        V = np.full((T, 1), 4.5e6)
        _, g, _ = gpu_grads(tr, dt0, dE0, V, np.zeros((T, 1)), *RES, target)
        out.append(g)
    for g in out[1:]:
        for k in g:
            assert normwise(g[k], out[0][k]) < 1e-12, k


C4_RES = (np.array([1e6]), np.array([1e9]), np.array([1.0]))  # broadband, stable over 500 turns


def c4_case(precision, T):
    n, S = 2_000_000, 1024
    _, rf, tr, dt0, dE0, target = make(n, S, T, precision=precision, K=50, intensity=3e9)
    V = np.full((T, 1), 4.5e6)
    L, g, _ = gpu_grads(tr, dt0, dE0, V, np.zeros((T, 1)), *C4_RES, target)
    return L, g, tr, dt0, dE0, target, V


def test_c4_size_fp64_against_finite_differences(cuda):
    """2e6 particles, 1024 slices, 500 turns, checkpoints every 50.  The map
    is piecewise smooth (linear deposition and interpolation put a kink
    wherever a particle crosses a bin centre), so a central difference
    measures the local derivative only while its perturbation moves few
    particles across bin centres over the remaining turns.  Measured error
    against step: within 6e-5 for steps 1e-7 .. 1e-9 (relative) for the
    resonator and the last 250 turns' voltages; for voltages 400 - 500
    turns before the loss it falls with the step (2.5 at 1e-7, 1e-2 at
    1e-8) down to ~5e-5 at 1e-9 .. 3e-9, below which rounding of the loss
    takes over.  The forward is bit-reproducible, so small steps carry no
    noise beyond rounding."""
    T = 500
    L, g, tr, dt0, dE0, target, V = c4_case("f64", T)
    n = tr.n

    def loss_gpu(V_, R_, fr_, Q_):
        with torch.no_grad():
            dt, dE, p = tr(torch.tensor(dt0, device="cuda"), torch.tensor(dE0, device="cuda"),
                           torch.tensor(V_, device="cuda"),
                           torch.zeros(T, 1, dtype=torch.float64, device="cuda"),
                           tr.impedance(*(torch.tensor(x, device="cuda") for x in (R_, fr_, Q_))))
            return float(bunch_loss(p, target, tr.bin_centers()))

    assert loss_gpu(V, *C4_RES) == loss_gpu(V, *C4_RES) == L
    R, fr, Q = C4_RES
    for kind, idx, step in (("V", (0, 0), 1e-9), ("V", (100, 0), 3e-9), ("V", (250, 0), 1e-7),
                            ("V", (499, 0), 1e-7), ("R", 0, 1e-7), ("fr", 0, 1e-7),
                            ("Q", 0, 1e-7)):
        a = {"V": V, "R": R, "fr": fr, "Q": Q}
        h = step * abs(a[kind][idx])
        up = {k: v.copy() for k, v in a.items()}
        dn = {k: v.copy() for k, v in a.items()}
        up[kind][idx] += h
        dn[kind][idx] -= h
        ref = (loss_gpu(up["V"], up["R"], up["fr"], up["Q"])
               - loss_gpu(dn["V"], dn["R"], dn["fr"], dn["Q"])) / (2 * h)
        assert abs(g[kind][idx] - ref) <= 1e-4 * abs(ref), (kind, idx, g[kind][idx], ref)
    assert n == 2_000_000


def test_c4_size_f32p64_gradient_against_fp64(cuda):
    """The chosen form's gradient against the FP64 (reference) gradient
    over 100 turns, where the two trajectories still agree closely; over
    500 turns float rounding of the coordinates separates individual
    trajectories and the difference grows to a few percent (reported by
    bench.py --workload c4)."""
    T = 100
    g64 = c4_case("f64", T)[1]
    g32 = c4_case("f32p64", T)[1]
    for k in ("V", "phi", "R", "fr", "Q"):
        assert normwise(g32[k], g64[k]) < 1e-2, (k, normwise(g32[k], g64[k]))
    for k in ("V", "R", "fr", "Q"):
        assert normwise(g32[k], g64[k]) < 1e-3, (k, normwise(g32[k], g64[k]))
