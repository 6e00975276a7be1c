"""The batched Bragg sweep workload: independent two-component bragg_ad runs
with uneven grids and random pulse parameters.

Draws (numpy ``default_rng(seed)``), per instance:

* grid: one of 1D N in {1024, 2048, 4096, 8192, 16384} on [-64, 64) or 2D
  {256^2, 512^2} on [-16, 16)^2, uniformly;
* peak Rabi frequency Omega ~ U[2, 20]  (laser Amp[0] = Omega / 2),
  detuning delta ~ U[-4, 4] (laser_domh[0]), g ~ U[0, 200] (all four GS
  entries), pulse length T ~ U[0.5, 3] (AMP_T Gaussian centred at T/2 with
  sigma T/6);
* fixed: laser_k[0] = 8 (k_L = 4), alpha = 1/2, state 1 a normalised
  Gaussian exp(-r^2/2), state 2 empty, header time 0.
"""
from __future__ import annotations

import numpy as np

from . import binfmt
from .engine import Laser

SIZES = [(1, 1024), (1, 2048), (1, 4096), (1, 8192), (1, 16384), (2, 256), (2, 512)]
BOX = {1: 128.0, 2: 32.0}


def draw(count: int, seed: int = 1, sizes=SIZES):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        dim, n = sizes[int(rng.integers(len(sizes)))]
        om, delta, g, T = rng.uniform(2, 20), rng.uniform(-4, 4), rng.uniform(0, 200), rng.uniform(0.5, 3)
        L = BOX[dim]
        h = binfmt.make_header(dim, [n] * dim, [-L / 2] * dim, [L / 2] * dim)
        kw = dict(Amp=[om / 2, om / 2], laser_k=[8.0, 0], laser_domh=[delta, 0])
        out.append(dict(header=h, alpha=0.5, gs=[g, g, g, g], kw=kw, laser=Laser.make(**kw), pulse=(T / 2, T / 6)))
    return out


def initial_state(h) -> np.ndarray:
    dim = int(h["nDims"])
    xs = np.meshgrid(*[binfmt.x_coords(h, a) for a in range(dim)], indexing="ij")
    p = np.exp(-0.5 * sum(x * x for x in xs)).astype(np.complex128)
    vol = float(np.prod([h[k] for k in ("dx", "dy")[:dim]]))
    return p / np.sqrt(vol * np.sum(np.abs(p) ** 2))


def pulse_values(t0: float, nk: int, tc: float, sigma: float, dt: float):
    """AMP_T at t1 of the nk potential steps of a block starting at header time t0."""
    t = t0 + 0.5 * dt
    F = []
    for j in range(nk):
        t1 = t + 0.5 * dt
        F.append(np.exp(-((t1 - tc) ** 2) / (2 * sigma * sigma)))
        t += dt if j < nk - 1 else 0.5 * dt
    return np.array(F)
