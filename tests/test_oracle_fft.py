"""Known-answer tests of the oracle's FP64 transform (oracle/fft_cpu.c).

(1) agreement with numpy's pocketfft for every power-of-two length the solver
uses and a non-power-of-two one; (2) the spectral second derivative of
exp(-x^2) is (4x^2-2)exp(-x^2), the check cft_1d_test.cpp:56-97 performs with
ft(-1), *(-k^2), ft(+1); (3) ft(-1) then ft(+1) is the identity (dk*dx = 2pi/N).
"""
import numpy as np
import pytest

from atus2_b200 import binfmt
from oracle.oracle import Oracle


@pytest.mark.parametrize("shape", [(2,), (8,), (64,), (128,), (4096,), (12,), (32, 16), (8, 16, 4), (16, 16, 16)])
def test_fft_matches_pocketfft(shape):
    rng = np.random.default_rng(3)
    dim = len(shape)
    h = binfmt.make_header(dim, shape, [-1.0] * dim, [1.0] * dim)
    o = Oracle(h, 1)
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    f = a.copy()
    o.fft_raw(f, -1)
    ref = np.fft.fftn(a)
    assert np.linalg.norm(f - ref) / np.linalg.norm(ref) < 1e-15 * max(4, np.log2(a.size))
    b = a.copy()
    o.fft_raw(b, +1)
    ref = np.fft.ifftn(a) * a.size
    assert np.linalg.norm(b - ref) / np.linalg.norm(ref) < 1e-15 * max(4, np.log2(a.size))


def test_spectral_laplacian_of_gaussian():
    N = 256
    h = binfmt.make_header(1, [N], [-10.0], [10.0])
    o = Oracle(h, 1)
    x = binfmt.x_coords(h, 0)
    k = binfmt.k_coords(h, 0)
    f = np.exp(-x * x).astype(np.complex128)
    o.ft(f, -1)
    f *= -k * k
    o.ft(f, +1)
    exact = (4 * x * x - 2) * np.exp(-x * x)
    assert np.abs(f - exact).max() < 1e-12


def test_round_trip_identity():
    h = binfmt.make_header(3, [16, 8, 32], [-4.0, -2.0, -8.0], [4.0, 2.0, 8.0])
    o = Oracle(h, 1)
    rng = np.random.default_rng(5)
    a = rng.standard_normal((16, 8, 32)) + 1j * rng.standard_normal((16, 8, 32))
    b = a.copy()
    o.ft(b, -1)
    o.ft(b, +1)
    assert np.abs(b - a).max() < 1e-14
