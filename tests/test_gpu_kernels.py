"""bmath-level CUDA kernels vs the CPU oracle (through the C ABI).

Bars: FP64 coordinates within 1e-12 normwise of the oracle restatement;
slice counts bit-exact; FP32 within the reference's own single-precision
cross-backend tolerance (rtol 1e-5, unittests/test_compare_wraps.py:104-109)
expressed normwise.
"""
import numpy as np
import pytest
import torch

import cpu_oracle as o
from conftest import golden, normwise
from blond_b200 import bmath as bm

pytestmark = pytest.mark.gpu

T_C = 2.5e-9


def _bunch(n, dtype=np.float64, seed=0):
    rng = np.random.default_rng(seed)
    dt = (T_C + 0.4e-9 * rng.standard_normal(n)).astype(dtype)
    dE = (2.3e7 * rng.standard_normal(n)).astype(dtype)
    return dt, dE


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _tol(dtype):
    return 1e-12 if dtype == np.float64 else 1e-5


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", [1, 2, 1001, 200003])
def test_kick(cuda, dtype, n):
    dt, dE = _bunch(n, dtype)
    V, om, ph = [4.5e6, 0.45e6], [1.2579e9, 5.0316e9], [0.1, np.pi]
    gdt, gdE = _dev(dt), _dev(dE)
    bm.kick(gdt, gdE, V, om, ph, 1.0, 2, -1234.5)
    o.kick(dt, dE, V, om, ph, 1.0, -1234.5)
    assert normwise(gdE.cpu().numpy(), dE) < _tol(dtype)
    np.testing.assert_array_equal(gdt.cpu().numpy(), dt)


def test_kick_sine_against_numpy(cuda):
    """The FP64 kick's sine (Cody-Waite reduction by pi, odd polynomial on
    [-pi/2, pi/2]): a kick with V = 1, omega = 1, phi = 0, charge 1 from
    dE = 0 leaves exactly sin(dt) in dE.  Against numpy's sine over the RF
    phase's range and far beyond (to 3e8 rad): within 4e-16 absolute (two
    units in the last place of 1); to 1e12 rad within 2e-13 (the reduction's
    roundings grow with |x|); NaN and inf give NaN."""
    rng = np.random.default_rng(11)
    x = np.concatenate([rng.uniform(-4, 4, 100000), rng.uniform(-1e3, 1e3, 100000),
                        rng.uniform(-1e6, 1e6, 20000), rng.uniform(9e6, 2e7, 1000),
                        rng.uniform(-3e8, 3e8, 1000),
                        [0.0, -0.0, np.pi, -np.pi / 2, 1e-300, 5e-324, 1e7, 3e8]])
    far = np.concatenate([rng.uniform(1e9, 1e12, 1000), -rng.uniform(1e9, 1e12, 1000)])
    special = np.array([np.nan, np.inf, -np.inf])
    dt = _dev(np.concatenate([x, far, special]))
    dE = torch.zeros_like(dt)
    bm.kick(dt, dE, [1.0], [1.0], [0.0], 1.0, 1, 0.0)
    got = dE.cpu().numpy()
    n, m = len(x), len(far)
    assert np.max(np.abs(got[:n] - np.sin(x))) <= 4e-16
    assert np.max(np.abs(got[n:n + m] - np.sin(far))) <= 2e-13
    assert np.all(np.isnan(got[n + m:]))


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("solver", [0, 1, 2])
@pytest.mark.parametrize("order", [0, 1, 2])
def test_drift(cuda, dtype, solver, order):
    dt, dE = _bunch(30011, dtype, seed=1)
    par = [2.3e-5, 1.0, order, 1.786e-3, 2.1e-4, -3.3e-5, 1 / 18**2, 1.1e-4,
           -2.0e-5, 0.99935, 26.017e9]
    gdt, gdE = _dev(dt), _dev(dE)
    bm.drift(gdt, gdE, ["simple", "legacy", "exact"][solver], *par)
    o.drift(dt, dE, solver, *par)
    # the drift has no transcendental but sqrt (correctly rounded on both
    # sides) and is evaluated without FMA contraction in the reference's
    # operation order: bit-identical to the oracle
    np.testing.assert_array_equal(gdt.cpu().numpy(), dt)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("S", [1, 100, 1000, 2049, 16384, 70000])
def test_slice_beam_exact(cuda, dtype, S):
    dt, _ = _bunch(300007, dtype, seed=2)
    cl, cr = T_C - 1.25e-9, T_C + 1.25e-9
    out = torch.full((S,), 7.0, dtype=torch.from_numpy(dt).dtype, device="cuda")
    bm.slice_beam(_dev(dt), out, cl, cr)
    np.testing.assert_array_equal(out.cpu().numpy(), o.histogram(dt, cl, cr, S))


def test_slice_beam_edge_cases(cuda):
    S, cl, cr = 64, 0.0, 64.0
    edges = np.arange(0, 65, dtype=np.float64)  # exactly on every bin edge
    special = np.array([np.nan, np.inf, -np.inf, -1e300, 1e300, -0.0, 63.999999,
                        64.0, -1e-300])
    same = np.full(100003, 17.5)  # all in one bin: atomic contention
    for dt in (edges, special, same, np.zeros(0)):
        out = torch.zeros(S, dtype=torch.float64, device="cuda")
        bm.slice_beam(_dev(dt) if len(dt) else torch.zeros(0, dtype=torch.float64,
                                                           device="cuda"),
                      out, cl, cr)
        np.testing.assert_array_equal(out.cpu().numpy(), o.histogram(dt, cl, cr, S))


def test_slice_beam_reference_goldens(cuda):
    """The exact counts of unittests/beam_profile/test_beam_profile_object.py."""
    g = golden("profile_golden.npz")
    gdt = _dev(g["dt"])
    for S, cuts, ref in ((100, g["cuts1"], g["counts1"]), (200, g["cuts2"], g["counts2"])):
        out = torch.zeros(S, dtype=torch.float64, device="cuda")
        bm.slice_beam(gdt, out, *cuts)
        np.testing.assert_array_equal(out.cpu().numpy(), ref)
    out = torch.zeros(150, dtype=torch.float64, device="cuda")
    bm.slice_smooth(gdt, out, *g["cuts3"])
    np.testing.assert_allclose(out.cpu().numpy(), g["smooth3"], rtol=1e-6, atol=1e-9)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("S", [100, 1024, 40000])
def test_slice_smooth(cuda, dtype, S):
    dt, _ = _bunch(100003, dtype, seed=3)
    cl, cr = T_C - 1.25e-9, T_C + 1.25e-9
    out = torch.zeros(S, dtype=torch.from_numpy(dt).dtype, device="cuda")
    bm.slice_smooth(_dev(dt), out, cl, cr)
    ref = o.smooth_histogram(dt, cl, cr, S)
    assert normwise(out.cpu().numpy(), ref) < (1e-12 if dtype == np.float64 else 1e-5)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("S", [2, 257, 16384])
def test_linear_interp_kick(cuda, dtype, S):
    dt, dE = _bunch(100003, dtype, seed=4)
    edges = np.linspace(T_C - 1.25e-9, T_C + 1.25e-9, S + 1).astype(dtype)
    bc = ((edges[:-1] + edges[1:]) / 2).astype(dtype)
    V = (1e5 * np.sin(np.linspace(0, 7, S)) + 3e4).astype(dtype)
    gdt, gdE = _dev(dt), _dev(dE)
    bm.linear_interp_kick(gdt, gdE, V, bc, 1.0, -77.0)
    o.linear_interp_kick(dt, dE, V, bc, 1.0, -77.0)
    assert normwise(gdE.cpu().numpy(), dE) < _tol(dtype)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_rf_volt_comp(cuda, dtype):
    bc = np.linspace(T_C - 1.25e-9, T_C + 1.25e-9, 1000).astype(dtype)
    V, om, ph = [4.5e6, 0.45e6], [1.2579e9, 5.0316e9], [0.1, np.pi]
    out = bm.rf_volt_comp(V, om, ph, _dev(bc))
    assert normwise(out.cpu().numpy(), o.rf_volt_comp(V, om, ph, bc)) < _tol(dtype)


def test_fast_resonator(cuda):
    freq = np.fft.rfftfreq(16384, 2.5e-9 / 16384)
    R, Q, fr = [5e6, 1e5, 3e4], [1.0, 200.0, 3e4], [1e9, 200e6, 1.4e9]
    Z = bm.fast_resonator(np.array(R), np.array(Q), freq, np.array(fr)).cpu().numpy()
    ref = o.fast_resonator(R, Q, freq, fr)
    assert normwise(Z.real, ref.real) < 1e-14 and normwise(Z.imag, ref.imag) < 1e-14
    assert Z[0] == 0


def test_bad_arguments_raise(cuda):
    from blond_b200 import BlondB200Error
    dt = torch.zeros(10, dtype=torch.float64, device="cuda")
    with pytest.raises(BlondB200Error):
        bm.kick(dt, dt.clone(), [1.0] * 65, [1.0] * 65, [0.0] * 65, 1.0, 65, 0.0)
    with pytest.raises(TypeError):
        bm.kick(dt.cpu(), dt.cpu(), [1.0], [1.0], [0.0], 1.0, 1, 0.0)
    with pytest.raises(BlondB200Error):
        bm.rfft(torch.zeros(5000, dtype=torch.float64, device="cuda"), 5003 * 3)
