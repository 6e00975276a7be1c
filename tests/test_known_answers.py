"""Known answers of the split-step path, checked on the oracle (CPU) and on
the CUDA path (-m gpu) with the same calls: a free Gaussian packet against
its closed form, the linear harmonic-oscillator ground state and its mu,
two-level Rabi oscillations under uniform coupling, norm conservation of the
unitary steps, and (GPU only) the field transform against cuFFT through
torch.fft.  The reference ships no test that pins results; these fix the
physics independently of any implementation.
"""
import math

import numpy as np
import pytest

from atus2_b200 import binfmt
from oracle.oracle import Laser as OLaser
from oracle.oracle import Oracle
from replay import KIND_BRAGG_AD, KIND_NL

ENGINES = [pytest.param("oracle"), pytest.param("gpu", marks=pytest.mark.gpu)]


def _engine(kind, h, ncomp):
    """(engine, its Laser type) on header h."""
    if kind == "oracle":
        return Oracle(h, ncomp), OLaser
    from atus2_b200 import PREC_FP64, Laser, Solver

    return Solver(h, ncomp, PREC_FP64), Laser


def _grid(dim, n, L):
    return binfmt.make_header(dim, n, [-L / 2] * dim, [L / 2] * dim)


@pytest.mark.parametrize("engine", ENGINES)
def test_free_gaussian_packet(engine):
    """g = 0, V = 0, alpha = 1/2 (H = -d^2/dx^2 / 2): psi0 = exp(-x^2/(2 s^2)
    + i k0 x) evolves to sqrt(s^2/a) exp((s^2 k0 + i x)^2/(2a) - s^2 k0^2/2),
    a = s^2 + i t.  The kinetic step is exact in k-space, so 2000 steps of
    1024 points on [-64, 64) match the closed form to FFT rounding."""
    h = _grid(1, [1024], 128.0)
    x = binfmt.x_coords(h, 0)
    s2, k0 = 4.0, 2.0
    psi0 = np.exp(-x * x / (2 * s2) + 1j * k0 * x)
    e, _ = _engine(engine, h, 1)
    e.set_psi(0, psi0)
    e.set_alpha(0, [0.5])
    e.set_gs([0.0])
    e.set_dt(1e-3)
    for _ in range(2):
        e.block(1000, KIND_NL)
    t = e.t
    assert abs(t - 2.0) < 1e-12
    a = s2 + 1j * t
    exact = np.sqrt(s2 / a) * np.exp((s2 * k0 + 1j * x) ** 2 / (2 * a) - s2 * k0 * k0 / 2)
    got = np.asarray(e.psi(0))
    assert np.linalg.norm(got - exact) / np.linalg.norm(exact) < 1e-11


@pytest.mark.parametrize("engine", ENGINES)
def test_harmonic_ground_state(engine):
    """g = 0, V = w^2 x^2 / 2, alpha = 1/2: the Sobolev descent ends at the
    Gaussian (w/pi)^(1/4) exp(-w x^2/2) with mu = w/2 (the mu formula of the
    descent, m_ar sum[-Re(psi* Lap psi) + V |psi|^2]).  The descent
    renormalises only while |N - 1| > 1e-5, so the state and mu are compared
    at the particle number N it ends with (mu = N w / 2 for g = 0)."""
    w = 1.5
    h = _grid(1, [128], 16.0)
    x = binfmt.x_coords(h, 0)
    e, _ = _engine(engine, h, 1)
    e.set_psi(0, np.exp(-0.3 * x * x).astype(np.complex128))
    e.set_potential(0, 0.5 * w * w * x * x)
    e.set_gs([0.0])
    e.sob_init([0.5], 0.01)
    it, res = e.sob_run(1e-20, 200000)
    assert res <= 1e-20
    psi = np.asarray(e.psi(0))
    n = float(np.vdot(psi, psi).real) * float(h["dx"])
    assert abs(n - 1.0) <= 1e-5
    ref = math.sqrt(n) * (w / math.pi) ** 0.25 * np.exp(-w * x * x / 2)
    psi = psi * np.exp(-1j * np.angle(psi[64]))
    assert np.linalg.norm(psi - ref) / np.linalg.norm(ref) < 1e-8
    assert abs(float(e.sob_mu()[0]) - n * w / 2) < 1e-10


@pytest.mark.parametrize("engine", ENGINES)
def test_two_level_rabi_oscillation(engine):
    """Uniform coupling (laser_k = laser_dk = domh = 0, g = 0, no detuning) on
    a uniform state: only k = 0 is populated, the kinetic step is the
    identity, and each bragg_ad step rotates the two states by Omega dt, so
    the populations are N cos^2(Omega t) and N sin^2(Omega t)."""
    h = _grid(1, [64], 16.0)
    psi0 = np.full(64, 1.0 / math.sqrt(16.0), dtype=np.complex128)
    e, LaserT = _engine(engine, h, 2)
    e.set_psi(0, psi0)
    e.set_psi(1, np.zeros_like(psi0))
    for c in range(2):
        e.set_alpha(c, [0.5])
    e.set_gs([0.0, 0.0, 0.0, 0.0])
    e.set_dt(1e-3)
    A = 3.0
    laser = LaserT.make(Amp=[A, A], laser_k=[0.0, 0.0], laser_dk=[0.0, 0.0], laser_domh=[0.0, 0.0],
                        phase=[0.0, 0.0], chirp_rate=[0.0, 0.0], chirp=0.0, beta=[0.0, 0.0, 0.0],
                        DeltaL=[0.0, 0.0, 0.0, 0.0])
    steps = 0
    for _ in range(3):
        e.block(100, KIND_BRAGG_AD, laser, np.ones(100))
        steps += 100
        ang = A * steps * 1e-3
        n0, n1 = e.particle_number(0), e.particle_number(1)
        assert abs(n0 - math.cos(ang) ** 2) < 1e-12
        assert abs(n1 - math.sin(ang) ** 2) < 1e-12


@pytest.mark.parametrize("engine", ENGINES)
def test_norm_conservation(engine):
    """Kinetic and potential steps are unitary: 200 nonlinear steps (g = 50,
    harmonic V) on 16 x 32 x 16 keep the particle number to 1e-12."""
    h = _grid(3, [16, 32, 16], 12.0)
    X = np.meshgrid(*[binfmt.x_coords(h, a) for a in range(3)], indexing="ij")
    r2 = sum(v * v for v in X)
    rng = np.random.default_rng(4)
    psi0 = np.exp(-0.5 * r2) * (1 + 0.1 * rng.standard_normal(r2.shape)) + 0j
    e, _ = _engine(engine, h, 1)
    e.set_psi(0, psi0)
    e.set_alpha(0, [0.5, 0.5, 0.5])
    e.set_gs([50.0])
    e.set_potential(0, 0.5 * r2)
    e.set_dt(1e-3)
    n0 = e.particle_number(0)
    e.block(200, KIND_NL)
    assert abs(e.particle_number(0) - n0) / n0 < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("n", [[4096], [32768], [2048, 64], [64, 512], [32, 64, 128]])
def test_field_transform_matches_cufft(n):
    """atus_ft forward against torch.fft.fftn (cuFFT) times the reference's
    forward scale (dx / sqrt(2 pi))^dim, FP64; register-staged, three-stage
    and four-step transforms included."""
    import torch

    from atus2_b200 import PREC_FP64, Solver

    dim = len(n)
    h = _grid(dim, n, 10.0)
    rng = np.random.default_rng(6)
    a = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    s = Solver(h, 1, PREC_FP64)
    s.set_psi(0, a)
    s.ft(0, -1)
    got = np.asarray(s.psi(0))
    s.close()
    scale = float(np.prod([float(h[f"d{ax}"]) for ax in "xyz"[:dim]])) / (2 * math.pi) ** (dim / 2)
    ref = torch.fft.fftn(torch.from_numpy(a).cuda()).cpu().numpy() * scale
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-14
