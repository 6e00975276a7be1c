"""Parity at the benchmark's own grid sizes.

The FP64 256^3 two-component Bragg step runs kernel instantiations that the
reduced-grid tests never reach (256-point register-staged passes: the
contiguous z pass with the two components meeting in shared memory, the
strided x kinetic pass and the strided y transforms), and the 2048^2 double
slit runs the long-pencil tile passes.  Here both run at full size against
the oracle (the C restatement of the reference, on all host cores).

Bars: FP64 relative L2 <= 1e-11 of the state and of every component holding
>= 10 % of the norm, particle numbers to 1e-11 relative; mixed precision
(complex64 fields, FP64 phase arguments) relative L2 <= 1e-5 over these step
counts.
"""
import math
import os

import numpy as np
import pytest

from atus2_b200 import PREC_FP64, PREC_MIXED, Laser, Solver, binfmt
from gpu_util import rel_l2
from oracle.oracle import Laser as OLaser
from oracle.oracle import Oracle
from replay import KIND_BRAGG_AD, KIND_NL, KIND_NL_IF, gaussian_pulse

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-11
MIXED_TOL = 1e-5
THREADS = os.cpu_count() or 1


def _grid(dim, n, L, t=0.0):
    return binfmt.make_header(dim, n, [-L / 2] * dim, [L / 2] * dim, t=t)


def _state_close(psi, ref, tol):
    tot = math.sqrt(sum(float(np.vdot(r, r).real) for r in ref))
    err = math.sqrt(sum(float(np.vdot(p - r, p - r).real) for p, r in zip(psi, ref)))
    assert err / tot < tol, (err / tot, tol)
    for p, r in zip(psi, ref):
        nr = math.sqrt(float(np.vdot(r, r).real))
        if nr >= 0.1 * tot:
            assert rel_l2(p, r) < tol


def _bragg256_setup(e):
    """The 256^3 Bragg workload on [-32,32)^3 loaded into engine e: state 1
    Thomas-Fermi (mu = 10, g = 100, omega = 1), state 2 empty, alpha = 1/2,
    g_ij = 100, dt = 1e-3."""
    h = _grid(3, [256] * 3, 64.0)
    x = binfmt.x_coords(h, 0)
    r2 = x[:, None, None] ** 2 + x[None, :, None] ** 2 + x[None, None, :] ** 2
    psi1 = np.sqrt(np.maximum(0.0, (10.0 - 0.5 * r2) / 100.0)).astype(np.complex128)
    del r2
    psi1 /= math.sqrt(float(h["dx"] * h["dy"] * h["dz"]) * float(np.vdot(psi1, psi1).real))
    e.set_psi(0, psi1)
    e.set_psi(1, np.zeros_like(psi1))
    for c in range(2):
        e.set_alpha(c, [0.5, 0.5, 0.5])
    e.set_gs([100.0] * 4)
    e.set_dt(1e-3)


# laser_k = 8, laser_domh = 16, Amp = 4 (peak Omega 8)
LASER_KW = dict(beta=[0, 0, 0], DeltaL=[0, 0, 0, 0], Amp=[4.0, 4.0], laser_k=[8.0, 0], laser_dk=[0, 0],
                laser_domh=[16.0, 0], phase=[0, 0], chirp_rate=[0, 0], chirp=0.0)
PULSE = gaussian_pulse(0.025, 2 * 0.012 ** 2)  # centred inside the 50 pulse steps
BRAGG_BLOCKS = [(KIND_BRAGG_AD, 25), (KIND_BRAGG_AD, 25), (KIND_NL_IF, 10)]


def _pulse_values(t0, nk):
    t = t0 + 0.5e-3
    out = []
    for _ in range(nk):
        out.append(PULSE(t + 0.5e-3))
        t += 1e-3
    return np.array(out)


def _run_bragg_blocks(e, laser):
    """Runs BRAGG_BLOCKS on e; yields after each block."""
    for kind, nk in BRAGG_BLOCKS:
        if kind == KIND_BRAGG_AD:
            e.block(nk, kind, laser, _pulse_values(e.t, nk))
        else:
            e.block(nk, kind, laser)
        yield kind


@pytest.fixture(scope="module")
def bragg256_oracle():
    """Oracle states (t, psi_1, psi_2, N_1, N_2) after the pulse and at the end."""
    h = _grid(3, [256] * 3, 64.0)
    o = Oracle(h, 2, threads=THREADS)
    _bragg256_setup(o)
    snaps = []
    for b, _ in enumerate(_run_bragg_blocks(o, OLaser.make(**LASER_KW))):
        if b in (1, len(BRAGG_BLOCKS) - 1):
            snaps.append((o.t, [o.psi(c).copy() for c in range(2)], [o.particle_number(c) for c in range(2)]))
    del o
    return snaps


@pytest.mark.parametrize("prec,tol", [(PREC_FP64, FP64_TOL), (PREC_MIXED, MIXED_TOL)])
def test_bragg_256cubed_against_oracle(bragg256_oracle, prec, tol):
    """50 bragg_ad steps (2 blocks of 25, a Gaussian pulse of peak 8 centred
    inside them) then 10 freeprop steps at 256^3 x 2 components."""
    s = Solver(_grid(3, [256] * 3, 64.0), 2, prec)
    _bragg256_setup(s)
    k = 0
    for b, _ in enumerate(_run_bragg_blocks(s, Laser.make(**LASER_KW))):
        if b in (1, len(BRAGG_BLOCKS) - 1):
            t, ref, n_ref = bragg256_oracle[k]
            k += 1
            assert s.t == t
            assert n_ref[1] > 1e-3  # the pulse moved population
            _state_close([s.psi(c) for c in range(2)], ref, tol)
            n_s = [s.particle_number(c) for c in range(2)]
            np.testing.assert_allclose(n_s, n_ref, rtol=(1e-11 if prec == PREC_FP64 else 1e-6))
    s.close()


def _slit_inputs():
    """2D double slit at full size: 2048^2 on [-64,64)^2, V = 200 on |x| < 0.5
    except slits |y -+ 4| < 1, packet sigma = 4 at x = -20 with kx = 8, g = 1,
    alpha = 1/2, dt = 5e-4."""
    h = _grid(2, [2048, 2048], 128.0)
    x = binfmt.x_coords(h, 0)[:, None]
    y = binfmt.x_coords(h, 1)[None, :]
    V = np.where((np.abs(x) < 0.5) & ~((np.abs(y - 4) < 1) | (np.abs(y + 4) < 1)), 200.0, 0.0)
    psi = np.exp(-((x + 20) ** 2 + y ** 2) / 32.0) * np.exp(8j * x)
    psi /= math.sqrt(float(h["dx"] * h["dy"]) * float(np.vdot(psi, psi).real))
    return h, psi, V


def _slit_setup(e, psi, V):
    e.set_psi(0, psi)
    e.set_alpha(0, [0.5, 0.5])
    e.set_gs([1.0])
    e.set_potential(0, V)
    e.set_dt(5e-4)


@pytest.fixture(scope="module")
def slit_oracle():
    """Oracle states after each of two blocks of 100 steps."""
    h, psi, V = _slit_inputs()
    o = Oracle(h, 1, threads=THREADS)
    _slit_setup(o, psi, V)
    snaps = []
    for _ in range(2):
        o.block(100, KIND_NL)
        snaps.append((o.t, o.psi(0).copy(), o.particle_number(0)))
    return snaps


@pytest.mark.parametrize("prec,tol", [(PREC_FP64, FP64_TOL), (PREC_MIXED, MIXED_TOL)])
def test_double_slit_2048_against_oracle(slit_oracle, prec, tol):
    """200 steps of the 2048^2 double slit in two blocks of 100."""
    h, psi, V = _slit_inputs()
    s = Solver(h, 1, prec)
    _slit_setup(s, psi, V)
    for t, ref, n_ref in slit_oracle:
        s.block(100, KIND_NL)
        assert s.t == t
        assert rel_l2(s.psi(0), ref) < tol
        # complex64 fields: the norm random-walks by ~1e-7 per 100 steps here
        # (measured over 10^4 steps: |drift| <= 6e-7)
        assert abs(s.particle_number(0) - n_ref) < (1e-12 if prec == PREC_FP64 else 1e-6)
    s.close()


def test_mixed_error_after_10k_steps_256():
    """The 256^3 Bragg workload at full length (5000 bragg_ad steps with the
    pulse, then 5000 freeprop steps), mixed against FP64 on the GPU: the
    measured bound of the complex64 form.  FP32 transform rounding random-
    walks at ~2-3.5e-7 per step (3.9e-5 after 10^4 steps), so the bar is
    5e-5 of the state and a norm drift below 1e-6; FP64 keeps the norm to
    1e-8 (the reference's eigen-form of the 2x2 step is unitary to ~1e-10
    per block here)."""
    import torch

    import bench

    res = bench.run_accuracy3(torch.cuda.Stream())
    assert res["mixed"]["rel_l2_vs_fp64"]["state"] < 5e-5, res
    assert abs(res["mixed"]["norm_drift"]) < 1e-6, res
    assert abs(res["fp64"]["norm_drift"]) < 1e-8, res
