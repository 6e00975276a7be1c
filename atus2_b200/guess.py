"""Learned initial guess for the Sobolev ground-state solver (sobmin).

Problem family: 3D grid on [-16, 16)^3, V = (x^2 + w_y^2 y^2 + w_z^2 z^2) / 2,
one component, N = 1, alpha = 1/2, interaction g; draws w_y, w_z ~ U[0.5, 4],
g ~ log-uniform on [10, 2000].

The guess of a draw is the Hermite expansion

    psi(x, y, z) = sum_{a,b,c in {0,2,4,6}} C[a/2, b/2, c/2] phi_a(x/lx) phi_b(y/ly) phi_c(z/lz)

(phi_n the orthonormal Hermite functions, divided by sqrt(l)), with basis
lengths l from the draw itself -- l^2 = 1/w + (R/3)^2, the oscillator length
and a third of the Thomas-Fermi radius R = sqrt(2 mu_TF)/w -- and the 64
coefficients C predicted by an MLP from (w_y, w_z, log g) scaled to O(1).
The network trains (atus_guess_train, hand-written CUDA kernels) on the
coefficients of ground states that plain sobmin itself computed: the
projections of each converged state on the basis.  Plain sobmin from the
Thomas-Fermi guess stays the fallback; the converged residual and chemical
potential tell how good the learned guess was.

    python -m atus2_b200.guess generate --count 256 --out atus2_b200/data/sob_train_64.npz
    python -m atus2_b200.guess evaluate --held-out 200 --seed 2 --out <file.json>

The guess seeds sobmin through a small box (solve_learned): the descent runs
first on a box with the full grid's spacing that just holds the condensate,
from the decoded guess, and its converged state, embedded in the full box,
starts the descent there.
"""
from __future__ import annotations

import argparse
import ctypes as C
import concurrent.futures as cf
import json
import math
import os
import time

import numpy as np

from . import binfmt
from .engine import PREC_FP64, Solver, load_library

NIN, NOUT, NPARAM = 3, 64, 8576
L_BOX = 32.0
STEP = 4e-4       # fixed Sobolev step: stable for the largest corner potential of the family
EPS = 1e-10       # residual target (the reference's squared-norm residual)
ALPHA = 0.5
HERE = os.path.dirname(os.path.abspath(__file__))
TRAIN_FILE = os.path.join(HERE, "data", "sob_train_64.npz")


def header(n: int):
    return binfmt.make_header(3, [n] * 3, [-L_BOX / 2] * 3, [L_BOX / 2] * 3)


def draw(count: int, seed: int):
    rng = np.random.default_rng(seed)
    wy = rng.uniform(0.5, 4.0, count)
    wz = rng.uniform(0.5, 4.0, count)
    g = np.exp(rng.uniform(math.log(10.0), math.log(2000.0), count))
    return np.stack([wy, wz, g], axis=1)


def features(p) -> np.ndarray:
    p = np.atleast_2d(np.asarray(p, dtype=np.float64))
    c = 0.5 * (math.log(10.0) + math.log(2000.0))
    h = 0.5 * (math.log(2000.0) - math.log(10.0))
    return np.stack([(p[:, 0] - 2.25) / 1.75, (p[:, 1] - 2.25) / 1.75, (np.log(p[:, 2]) - c) / h], axis=1)


def mu_tf(wy: float, wz: float, g: float) -> float:
    """Thomas-Fermi chemical potential of N = 1 in the trap (1, wy, wz):
    N = (8 pi / 15) (2 mu)^{3/2} mu / (g wx wy wz)."""
    return (15.0 * g * wy * wz / (8.0 * math.pi * 2.0 * math.sqrt(2.0))) ** 0.4


def scales(wy: float, wz: float, g: float) -> np.ndarray:
    mu = mu_tf(wy, wz, g)
    w = np.array([1.0, wy, wz])
    R = np.sqrt(2.0 * mu) / w
    return np.sqrt(1.0 / w + (R / 3.0) ** 2)


def hermite_rows(n: int, dx: float, l: float) -> np.ndarray:
    """phi_n(x/l)/sqrt(l), n = 0, 2, 4, 6, at x_i = (i - n/2) dx: shape (4, n)."""
    x = (np.arange(n) - n // 2) * dx
    u = x / l
    out = np.zeros((4, n))
    pm, pc = np.zeros(n), math.pi ** -0.25 / math.sqrt(l) * np.exp(-0.5 * u * u)
    for q in range(7):
        if q % 2 == 0:
            out[q // 2] = pc
        pn = math.sqrt(2.0 / (q + 1)) * u * pc - math.sqrt(q / (q + 1)) * pm
        pm, pc = pc, pn
    return out


def project(psi: np.ndarray, h, sc) -> np.ndarray:
    """Least-squares coefficients of psi (real part) on the basis sampled on
    the grid: the separable normal equations, one 4 x 4 Gram matrix per axis
    (the sampled functions are orthonormal only on fine grids)."""
    n = psi.shape
    B = [hermite_rows(n[a], float(h[f"d{'xyz'[a]}"]), sc[a]) for a in range(3)]
    r = np.einsum("ijk,ai,bj,ck->abc", psi.real, B[0], B[1], B[2])
    Gi = [np.linalg.inv(b @ b.T) for b in B]
    return np.einsum("abc,pa,qb,rc->pqr", r, Gi[0], Gi[1], Gi[2]).ravel()


def decode(coef, h, sc) -> np.ndarray:
    n = [int(h[f"nDim{a}"]) for a in "XYZ"]
    B = [hermite_rows(n[a], float(h[f"d{'xyz'[a]}"]), sc[a]) for a in range(3)]
    return np.einsum("abc,ai,bj,ck->ijk", np.asarray(coef).reshape(4, 4, 4), B[0], B[1], B[2])


def potential(h, wy, wz):
    x, y, z = np.meshgrid(*[binfmt.x_coords(h, a) for a in range(3)], indexing="ij")
    return 0.5 * (x * x + wy * wy * y * y + wz * wz * z * z)


def tf_guess(h, V, g):
    """sqrt(max(0, (mu - V)/g)) with mu set by N = 1 on the grid (bisection)."""
    dv = float(h["dx"] * h["dy"] * h["dz"])
    lo, hi = 0.0, float(V.max()) + 1e3 * g
    for _ in range(200):
        mu = 0.5 * (lo + hi)
        if np.sum(np.maximum(0.0, mu - V)) / g * dv > 1.0:
            hi = mu
        else:
            lo = mu
    return np.sqrt(np.maximum(0.0, (mu - V) / g)).astype(np.complex128)


def solve(n, wy, wz, g, coef=None, eps=EPS, max_iter=200000):
    """Plain sobmin from the Thomas-Fermi guess (coef None) or from the
    learned guess; returns (psi, iterations, residual, seconds, mu)."""
    h = header(n)
    V = potential(h, wy, wz)
    s = Solver(h, 1, PREC_FP64)
    if coef is None:
        s.set_psi(0, tf_guess(h, V, g))
    else:
        s.guess_decode(0, coef, scales(wy, wz, g))
    s.set_potential(0, V)
    s.set_gs([g])
    s.sob_init([ALPHA], STEP)
    s.synchronize()
    t0 = time.perf_counter()
    it, res = s.sob_run(eps, max_iter)
    s.synchronize()
    dt = time.perf_counter() - t0
    mu = float(s.sob_mu()[0])
    psi = s.psi(0)
    s.close()
    return psi, it, res, dt, mu


def mu_normalized(n, wy, wz, g, psi):
    """mu (the descent's formula) of `psi` scaled to particle number 1."""
    h = header(n)
    s = Solver(h, 1, PREC_FP64)
    nrm = (L_BOX / n) ** 3 * np.vdot(psi, psi).real
    s.set_psi(0, psi / math.sqrt(nrm))
    s.set_potential(0, potential(h, wy, wz))
    s.set_gs([g])
    s.sob_init([ALPHA], STEP)
    mu = float(s.sob_mu()[0])
    s.close()
    return mu


def small_box(n: int, wy: float, wz: float, g: float, margin: float = 3.0):
    """Points per axis of the smallest grid with the full grid's spacing that
    holds the condensate of a draw: twice its Thomas-Fermi radius plus
    `margin` oscillator lengths on each side, rounded up to a power of two
    (at least 16, at most n)."""
    mu = mu_tf(wy, wz, g)
    dx = L_BOX / n
    out = []
    for w in (1.0, wy, wz):
        half = math.sqrt(2.0 * mu) / w + margin / math.sqrt(w)
        m = 16
        while m < n and m * dx < 2.0 * half:
            m *= 2
        out.append(min(m, n))
    return out


def solve_learned(n, wy, wz, g, coef, eps=EPS, margin=3.0, max_iter=400000):
    """sobmin seeded by the learned guess: the guess decoded on the small box
    of the draw (small_box: the full grid's spacing, just large enough for the
    condensate), the descent there to eps, the converged state embedded in
    the full box (atus_embed), and the descent on the full box to eps from
    there.  The slow modes of the fixed-step descent are the condensate's own
    low modes, which the small box holds exactly at a fraction of the cost
    per iteration; on the full box only the tails outside the small box are
    left.  A draw whose small box is the full box runs plain sobmin from the
    learned guess.  Returns (psi, [iterations small, full], residual, seconds,
    mu, small-box points); the seconds cover both descents and the embedding
    (the grids and potentials are set up before the clock starts, as in
    solve())."""
    ns = small_box(n, wy, wz, g, margin)
    hf = header(n)
    f = Solver(hf, 1, PREC_FP64)
    f.set_potential(0, potential(hf, wy, wz))
    f.set_gs([g])
    f.sob_init([ALPHA], STEP)
    s = None
    if ns != [n, n, n]:
        hs = binfmt.make_header(3, ns, [-0.5 * m * L_BOX / n for m in ns], [0.5 * m * L_BOX / n for m in ns])
        s = Solver(hs, 1, PREC_FP64)
        s.guess_decode(0, coef, scales(wy, wz, g))
        s.set_potential(0, potential(hs, wy, wz))
        s.set_gs([g])
        s.sob_init([ALPHA], STEP)
        s.synchronize()
    else:
        f.guess_decode(0, coef, scales(wy, wz, g))
    f.synchronize()
    t0 = time.perf_counter()
    iters = [0]
    if s is not None:
        it, _ = s.sob_run(eps, max_iter)
        iters = [it]
        f.embed_from(s)
    it, res = f.sob_run(eps, max_iter)
    iters.append(it)
    f.synchronize()
    dt = time.perf_counter() - t0
    mu = float(f.sob_mu()[0])
    psi = f.psi(0)
    f.close()
    if s is not None:
        s.close()
    return psi, iters, res, dt, mu, ns


def generate(count: int, seed: int, n: int = 64, workers: int = 8):
    """Training set: plain-sobmin ground states of `count` draws at n^3,
    projected on their bases."""
    P = draw(count, seed)

    def one(k):
        wy, wz, g = P[k]
        psi, it, res, dt, mu = solve(n, wy, wz, g)
        return project(psi, header(n), scales(wy, wz, g)), it, res, mu

    with cf.ThreadPoolExecutor(workers) as ex:
        out = list(ex.map(one, range(count)))
    coef = np.stack([o[0] for o in out])
    return dict(params=P, coef=coef, iters=np.array([o[1] for o in out]), res=np.array([o[2] for o in out]),
                mu=np.array([o[3] for o in out]), n=n, seed=seed, step=STEP, eps=EPS)


# ------------------------------------------------------------------ network (C ABI)
def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def init_params(seed: int) -> np.ndarray:
    p = np.zeros(NPARAM)
    _check(load_library().atus_guess_init(C.c_uint64(seed), _dp(p)), "guess_init")
    return p


def _check(r, what):
    if r != 0:
        raise RuntimeError(f"{what} failed: {r}")


def grad(params, X, Y):
    X = np.ascontiguousarray(X, dtype=np.float64)
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    p = np.ascontiguousarray(params, dtype=np.float64)
    g = np.zeros(NPARAM)
    loss = np.zeros(1)
    _check(load_library().atus_guess_grad(_dp(p), _dp(X), _dp(Y), len(X), _dp(loss), _dp(g)), "guess_grad")
    return float(loss[0]), g


def train(X, Y, epochs=20000, lr=2e-3, seed=0, params=None):
    X = np.ascontiguousarray(X, dtype=np.float64)
    Y = np.ascontiguousarray(Y, dtype=np.float64)
    p = init_params(seed) if params is None else np.array(params, dtype=np.float64)
    hist = np.zeros(epochs)
    _check(load_library().atus_guess_train(_dp(p), _dp(X), _dp(Y), len(X), int(epochs), float(lr), _dp(hist)),
           "guess_train")
    return p, hist


def predict(params, X):
    X = np.ascontiguousarray(X, dtype=np.float64)
    p = np.ascontiguousarray(params, dtype=np.float64)
    out = np.zeros((len(X), NOUT))
    _check(load_library().atus_guess_predict(_dp(p), _dp(X), len(X), _dp(out)), "guess_predict")
    return out


# Coefficients are trained in units of their spread over the training set.
def coef_stats(coef):
    return coef.mean(axis=0), coef.std(axis=0) + 1e-12


def evaluate(count: int, seed: int, n: int = 128, train_epochs: int = 20000):
    """The learned guess on `count` held-out draws (seed `seed`): plain sobmin
    from the Thomas-Fermi guess against solve_learned, both to EPS; per draw
    iterations, seconds, mu and the particle number of the final state
    (the reference's descent renormalises only when |N - 1| > 1e-5, so two
    converged runs end at slightly different N and mu; dmu_normalized
    compares the two states scaled to N = 1)."""
    d = np.load(TRAIN_FILE)
    m, sd = coef_stats(d["coef"])
    params, hist = train(features(d["params"]), (d["coef"] - m) / sd, epochs=train_epochs, lr=2e-3)
    H = draw(count, seed)
    pred = predict(params, features(H)) * sd + m
    rows = []
    dv = (L_BOX / n) ** 3
    for k, (wy, wz, g) in enumerate(H):
        psi_p, it_p, res_p, t_p, mu_p = solve(n, wy, wz, g)
        psi_l, it_l, res_l, t_l, mu_l, ns = solve_learned(n, wy, wz, g, pred[k])
        rows.append(dict(w_y=float(wy), w_z=float(wz), g=float(g), iters_plain=int(it_p), s_plain=t_p, mu_plain=mu_p,
                         N_plain=float(dv * np.vdot(psi_p, psi_p).real), iters_learned=[int(i) for i in it_l],
                         s_learned=t_l, mu_learned=mu_l, N_learned=float(dv * np.vdot(psi_l, psi_l).real),
                         small_box=ns, speedup=t_p / t_l, dmu=abs(mu_l - mu_p),
                         dmu_normalized=abs(mu_normalized(n, wy, wz, g, psi_l) - mu_normalized(n, wy, wz, g, psi_p)),
                         rel_l2=float(np.linalg.norm(psi_l - psi_p) / np.linalg.norm(psi_p))))
        print(json.dumps(rows[-1]), flush=True)
    sp = np.array([r["speedup"] for r in rows])
    return dict(count=count, seed=seed, n=n, rows=rows, mean_speedup=float(sp.mean()),
                total_speedup=float(sum(r["s_plain"] for r in rows) / sum(r["s_learned"] for r in rows)),
                min_speedup=float(sp.min()), frac_ge_3=float((sp >= 3).mean()),
                max_dmu=float(max(r["dmu"] for r in rows)),
                max_dmu_normalized=float(max(r["dmu_normalized"] for r in rows)),
                training_loss=[float(hist[0]), float(hist[-1])])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["generate", "evaluate"])
    ap.add_argument("--count", type=int, default=256)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--n", type=int, default=64)
    ap.add_argument("--workers", type=int, default=8)
    ap.add_argument("--out", default=TRAIN_FILE)
    ap.add_argument("--held-out", type=int, default=200, help="evaluate: number of held-out draws (seed --seed)")
    a = ap.parse_args()
    if a.cmd == "evaluate":
        out = evaluate(a.held_out, a.seed)
        with open(a.out, "w") as f:
            json.dump(out, f)
        print(f"{a.held_out} draws: mean speed-up {out['mean_speedup']:.2f}, total {out['total_speedup']:.2f}, "
              f"min {out['min_speedup']:.2f}, >= 3x for {100 * out['frac_ge_3']:.0f} %, max |dmu| {out['max_dmu']:.2e}, "
              f"at N = 1 {out['max_dmu_normalized']:.2e}")
        return
    t0 = time.perf_counter()
    d = generate(a.count, a.seed, a.n, a.workers)
    os.makedirs(os.path.dirname(a.out), exist_ok=True)
    np.savez_compressed(a.out, **d)
    print(f"{a.count} ground states at {a.n}^3 in {time.perf_counter() - t0:.1f} s; "
          f"iterations {d['iters'].min()}..{d['iters'].max()}; residuals <= {d['res'].max():.2e}")


if __name__ == "__main__":
    main()
