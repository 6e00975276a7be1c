"""The learned sobmin guess: basis and network on the CPU; the CUDA training
kernels against the numpy restatement (oracle/mlp_oracle.py); and what a
trained network gains over the Thomas-Fermi start on held-out draws."""
import math

import numpy as np
import pytest

from atus2_b200 import guess
from oracle import mlp_oracle as mo

gpu = pytest.mark.gpu


def test_hermite_basis_is_orthonormal():
    B = guess.hermite_rows(512, 0.05, 1.3)
    G = B @ B.T * 0.05
    np.testing.assert_allclose(G, np.eye(4), atol=1e-10)


def test_project_inverts_decode():
    h = guess.header(48)
    sc = guess.scales(1.7, 2.9, 300.0)
    c = np.random.default_rng(0).standard_normal(64)
    back = guess.project(guess.decode(c, h, sc).astype(np.complex128), h, sc)
    np.testing.assert_allclose(back, c, atol=1e-8)


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = rng.standard_normal(mo.NP) * 0.2
    X, Y = rng.standard_normal((5, 3)), rng.standard_normal((5, 64))
    loss, g = mo.loss_grad(p, X, Y)
    for q in rng.integers(0, mo.NP, 25):
        e = np.zeros(mo.NP)
        e[q] = 1e-6
        fd = (mo.loss_grad(p + e, X, Y)[0] - mo.loss_grad(p - e, X, Y)[0]) / 2e-6
        assert abs(fd - g[q]) <= 1e-7 * max(1.0, abs(g[q]))


@gpu
def test_cuda_gradient_matches_oracle():
    rng = np.random.default_rng(2)
    p = guess.init_params(5)
    p[mo.NH * 3:mo.NH * 3 + mo.NH] = 0.1 * rng.standard_normal(mo.NH)  # nonzero biases too
    X, Y = rng.standard_normal((37, 3)), rng.standard_normal((37, 64))
    loss, g = guess.grad(p, X, Y)
    lo, go = mo.loss_grad(p, X, Y)
    assert abs(loss - lo) <= 1e-13 * lo
    assert np.linalg.norm(g - go) <= 1e-12 * np.linalg.norm(go)


@gpu
def test_cuda_adam_and_inference_match_oracle():
    rng = np.random.default_rng(3)
    X, Y = rng.standard_normal((20, 3)), rng.standard_normal((20, 64))
    p0 = guess.init_params(11)
    p, hist = guess.train(X, Y, epochs=30, lr=1e-3, params=p0)
    po, ho = mo.adam(p0, X, Y, 30, 1e-3)
    np.testing.assert_allclose(hist, ho, rtol=1e-11)
    assert np.linalg.norm(p - po) <= 1e-11 * np.linalg.norm(po)
    np.testing.assert_allclose(guess.predict(p, X), mo.forward(po, X)[0], rtol=1e-10, atol=1e-12)


@gpu
def test_decode_kernel_matches_host_expansion():
    from atus2_b200 import PREC_FP64, Solver

    h = guess.header(32)
    sc = guess.scales(1.2, 3.1, 80.0)
    c = np.random.default_rng(4).standard_normal(64)
    s = Solver(h, 1, PREC_FP64)
    s.guess_decode(0, c, sc)
    ref = guess.decode(c, h, sc)
    assert np.linalg.norm(s.psi(0) - ref) <= 1e-13 * np.linalg.norm(ref)


@gpu
def test_trained_guess_needs_fewer_iterations():
    """Train on plain-sobmin ground states (32^3, residual 1e-8) of 48 draws;
    on 3 held-out draws the learned start converges in fewer iterations than
    the Thomas-Fermi start, to the same chemical potential."""
    n, eps = 32, 1e-8
    P = guess.draw(48, 21)

    def one(k):
        wy, wz, g = P[k]
        psi, it, res, dt, mu = guess.solve(n, wy, wz, g, eps=eps)
        return guess.project(psi, guess.header(n), guess.scales(wy, wz, g))

    import concurrent.futures as cf

    with cf.ThreadPoolExecutor(8) as ex:
        coef = np.stack(list(ex.map(one, range(len(P)))))
    m, sd = guess.coef_stats(coef)
    params, hist = guess.train(guess.features(P), (coef - m) / sd, epochs=6000, lr=2e-3)
    assert hist[-1] < 0.05 * hist[0]
    H = guess.draw(3, 22)
    pred = guess.predict(params, guess.features(H)) * sd + m
    gains = []
    for k, (wy, wz, g) in enumerate(H):
        _, it_tf, _, _, mu_tf = guess.solve(n, wy, wz, g, eps=eps)
        _, it_nn, res_nn, _, mu_nn = guess.solve(n, wy, wz, g, coef=pred[k], eps=eps)
        print(f"draw {k}: TF {it_tf} iterations, learned {it_nn}; mu {mu_tf:.10f} / {mu_nn:.10f}")
        assert res_nn <= eps
        # both runs stop at residual 1e-8 (a squared norm): mu agrees to ~sqrt of it
        assert abs(mu_nn - mu_tf) <= 1e-4 * abs(mu_tf)
        gains.append(it_tf / it_nn)
    print("iteration ratios TF / learned:", gains)
    assert min(gains) > 1.0
