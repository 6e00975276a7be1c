"""Batched sweep (atus_batch_*): every instance of a batch computes the bragg_ad
run the oracle computes for the same parameters, whichever kernel variant the
size class runs with, before and after the autotuner."""
import numpy as np
import pytest

from atus2_b200 import PREC_FP64, PREC_MIXED, Batch, Laser, binfmt
from gpu_util import rel_l2
from oracle.oracle import Laser as OLaser
from oracle.oracle import Oracle
from replay import KIND_BRAGG_AD

pytestmark = pytest.mark.gpu

DT = 1e-3
FP64_TOL = 1e-11
MIXED_TOL = 1e-4


def _instances(seed, sizes):
    """Sweep parameters as the batched benchmark draws them: peak Rabi
    frequency U[2,20], detuning U[-4,4], g U[0,200], pulse length T U[0.5,3]
    (AMP_T centred at T/2 with sigma T/6)."""
    rng = np.random.default_rng(seed)
    out = []
    for dim, n in sizes:
        L = 64.0 if dim == 1 else 32.0
        h = binfmt.make_header(dim, [n] * dim, [-L / 2] * dim, [L / 2] * dim)
        om, delta, g, T = rng.uniform(2, 20), rng.uniform(-4, 4), rng.uniform(0, 200), rng.uniform(0.5, 3)
        kw = dict(Amp=[om / 2, om / 2], laser_k=[8.0, 0], laser_domh=[delta, 0])
        out.append(dict(header=h, alpha=0.5, gs=[g, g, g, g], kw=kw, laser=Laser.make(**kw), pulse=(T / 2, T / 6)))
    return out


def _psi0(h):
    dim = int(h["nDims"])
    xs = np.meshgrid(*[binfmt.x_coords(h, a) for a in range(dim)], indexing="ij")
    r2 = sum(x * x for x in xs)
    p = np.exp(-0.5 * r2).astype(np.complex128)
    vol = float(np.prod([h[k] for k in ("dx", "dy")[:dim]]))
    return p / np.sqrt(vol * np.sum(np.abs(p) ** 2))


def _pulse_values(t0, nk, tc, sigma):
    t = t0 + 0.5 * DT
    F = []
    for j in range(nk):
        t1 = t + 0.5 * DT
        F.append(np.exp(-((t1 - tc) ** 2) / (2 * sigma * sigma)))
        t += DT if j < nk - 1 else 0.5 * DT
    return np.array(F), t


def _oracle_runs(insts, blocks):
    res = []
    for d in insts:
        h = d["header"]
        o = Oracle(h, 2)
        o.set_psi(0, _psi0(h))
        o.set_psi(1, np.zeros_like(_psi0(h)))
        for c in range(2):
            o.set_alpha(c, [d["alpha"]] * int(h["nDims"]))
        o.set_gs(d["gs"])
        o.set_dt(DT)
        t = float(h["t"])
        for nk in blocks:
            F, t = _pulse_values(t, nk, *d["pulse"])
            o.block(nk, KIND_BRAGG_AD, OLaser.make(**d["kw"]), F)
        res.append((o.psi(0).copy(), o.psi(1).copy(), o.t))  # psi() is a live view into the oracle
    return res


def _check(b, insts, ref, tol):
    for i, (p0, p1, t) in enumerate(ref):
        assert abs(b.time(i) - t) < 1e-12
        got = np.stack([b.psi(i, 0), b.psi(i, 1)])
        want = np.stack([p0, p1])
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err < tol, (i, insts[i]["header"]["nDimX"], err)
        assert rel_l2(got[0], want[0]) < tol


@pytest.mark.parametrize("variant", ["0", "1", "2"])
def test_batch_fp64_matches_oracle(variant, monkeypatch):
    """FP64 batch: 1D lengths with both components resident and with one
    parked in L2, 2D register-staged and tile passes; every variant index."""
    monkeypatch.setenv("ATUS_BATCH_VARIANT", variant)
    sizes = [(1, 1024), (1, 2048), (1, 1024), (1, 8192), (2, 64), (2, 128), (2, 64)]
    insts = _instances(11, sizes)
    b = Batch(insts, PREC_FP64, DT)
    for i, d in enumerate(insts):
        b.set_psi(i, 0, _psi0(d["header"]))
        b.set_psi(i, 1, np.zeros_like(_psi0(d["header"])))
    b.run(40)
    b.run(25)
    _check(b, insts, _oracle_runs(insts, [40, 25]), FP64_TOL)


def test_batch_mixed_tuned_matches_oracle():
    """Mixed batch (complex64 fields, FP64 phase arguments) with the
    autotuner's choice, against the FP64 oracle."""
    sizes = [(1, 1024), (1, 16384), (1, 4096), (2, 64), (2, 256), (2, 512)]
    insts = _instances(12, sizes)
    b = Batch(insts, PREC_MIXED, DT)
    for i, d in enumerate(insts):
        b.set_psi(i, 0, _psi0(d["header"]))
        b.set_psi(i, 1, np.zeros_like(_psi0(d["header"])))
    b.run(30)
    b.tune(5)
    sched = b.schedule()
    print(sched)
    assert "probe ms" in sched
    b.run(30)
    _check(b, insts, _oracle_runs(insts, [30, 30]), MIXED_TOL)


@pytest.mark.parametrize("variant", ["0", "1"])
def test_batch_mixed_variants_match_oracle(variant, monkeypatch):
    """Mixed batch with each 2D variant forced: 512^2 register-staged or tile
    passes, 256^2 register-staged or tile passes."""
    monkeypatch.setenv("ATUS_BATCH_VARIANT", variant)
    sizes = [(2, 512), (2, 256), (1, 2048)]
    insts = _instances(13, sizes)
    b = Batch(insts, PREC_MIXED, DT)
    for i, d in enumerate(insts):
        b.set_psi(i, 0, _psi0(d["header"]))
        b.set_psi(i, 1, np.zeros_like(_psi0(d["header"])))
    b.run(40)
    _check(b, insts, _oracle_runs(insts, [40]), MIXED_TOL)
