"""Cluster FFT, irfft and one-turn induced voltage vs numpy (pocketfft, the
library the reference calls).  Bar: 1e-10 normwise (induced voltage), the
parity definition for this step; the transforms themselves reach ~1e-15."""
import numpy as np
import pytest
import torch

import cpu_oracle as o
from conftest import golden, normwise
from blond_b200 import bmath as bm

pytestmark = pytest.mark.gpu

# even 5-smooth lengths (cluster path), incl. next_regular values such as
# 1080, and lengths the direct-DFT path handles (odd / prime factor > 5)
SMOOTH = [2, 4, 16, 32, 60, 1080, 2048, 3000, 4096, 8192, 16384, 32768, 65536, 131072]
DIRECT = [1, 7, 1001, 1014, 4096 - 2]


@pytest.mark.parametrize("n", SMOOTH + DIRECT)
def test_rfft_irfft(cuda, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(max(1, n - 3))
    X = bm.rfft(x, n).cpu().numpy()
    ref = np.fft.rfft(x, n)
    assert normwise(X, ref) < 1e-13
    Y = rng.standard_normal(n // 2 + 1) + 1j * rng.standard_normal(n // 2 + 1)
    y = bm.irfft(Y, n).cpu().numpy()
    assert normwise(y, np.fft.irfft(Y, n)) < 1e-13


def test_rfft_zero_pads_and_truncates(cuda):
    x = np.arange(10.0)
    assert normwise(bm.rfft(x, 16).cpu().numpy(), np.fft.rfft(x, 16)) < 1e-14
    assert normwise(bm.rfft(x, 6).cpu().numpy(), np.fft.rfft(x, 6)) < 1e-14


@pytest.mark.parametrize("S,n_fft", [(16, 16), (16, 1080), (100, 100), (1024, 1024),
                                     (512, 2048), (4096, 4096), (3000, 8192), (8192, 8192),
                                     (10000, 16384), (16384, 16384), (65536, 65536)])
def test_induced_voltage_1turn(cuda, S, n_fft):
    rng = np.random.default_rng(S)
    prof = np.floor(1000 * np.exp(-np.linspace(-3, 3, S) ** 2) + rng.random(S))
    freq = np.fft.rfftfreq(n_fft, 2.5e-9 / S)
    Z = o.fast_resonator([5e6], [1.0], freq, [1e9]) / (2.5e-9 / S)
    v = bm.induced_voltage_1turn(prof, Z, n_fft, 1.6e-9, S).cpu().numpy()
    ref = -(1.6e-9 * np.fft.irfft(Z * np.fft.rfft(prof, n_fft)))[:S]
    assert normwise(v, ref) < 1e-10


def test_induced_voltage_reference_fixture(cuda):
    """Golden n_fft=1080 impedance of the reference (frequency_resolution
    3e6 case) applied to a profile."""
    g = golden("nfft_known.npz")
    Z = g["freq_res3e6_impedance"]
    prof = np.floor(50 * np.exp(-np.linspace(-2, 2, 16) ** 2))
    v = bm.induced_voltage_1turn(prof, Z, 1080, 1.0, 1067).cpu().numpy()
    ref = -np.fft.irfft(Z * np.fft.rfft(prof, 1080))[:1067]
    assert normwise(v, ref) < 1e-10
