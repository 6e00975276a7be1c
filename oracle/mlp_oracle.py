"""CPU restatement of the learned-guess network.

TEST INFRASTRUCTURE ONLY: imported by tests/ and bench.py checks, never by
the ``atus2_b200`` package.

The network of atus2_b200/csrc/guess.cu in numpy, FP64: inputs (3), two tanh
layers of 64, 64 linear outputs; loss = mean over samples and outputs of
(out - target)^2; Adam with bias correction.  The reference has no such
network: this file checks the project's own CUDA training kernels (forward,
backward and update) against plain numpy on the same inputs.
"""
from __future__ import annotations

import numpy as np

NI, NH, NO = 3, 64, 64
NP = NH * NI + NH + NH * NH + NH + NO * NH + NO


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + NH * NI].reshape(NH, NI); o += NH * NI
    b1 = p[o:o + NH]; o += NH
    W2 = p[o:o + NH * NH].reshape(NH, NH); o += NH * NH
    b2 = p[o:o + NH]; o += NH
    W3 = p[o:o + NO * NH].reshape(NO, NH); o += NO * NH
    b3 = p[o:o + NO]
    return W1, b1, W2, b2, W3, b3


def forward(p, X):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    h1 = np.tanh(X @ W1.T + b1)
    h2 = np.tanh(h1 @ W2.T + b2)
    return h2 @ W3.T + b3, h1, h2


def loss_grad(p, X, Y):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    out, h1, h2 = forward(p, X)
    B = X.shape[0]
    r = out - Y
    loss = float(np.sum(r * r) / (B * NO))
    d3 = 2.0 * r / (B * NO)
    gW3 = d3.T @ h2
    gb3 = d3.sum(axis=0)
    d2 = (d3 @ W3) * (1.0 - h2 * h2)
    gW2 = d2.T @ h1
    gb2 = d2.sum(axis=0)
    d1 = (d2 @ W2) * (1.0 - h1 * h1)
    gW1 = d1.T @ X
    gb1 = d1.sum(axis=0)
    return loss, np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])


def adam(p, X, Y, epochs, lr, b1=0.9, b2=0.999, eps=1e-12):
    p = np.array(p, dtype=np.float64)
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    hist = []
    for e in range(1, epochs + 1):
        loss, g = loss_grad(p, X, Y)
        hist.append(loss)
        m = b1 * m + (1 - b1) * g
        v = b2 * v + (1 - b2) * g * g
        p = p - lr * (m / (1 - b1 ** e)) / (np.sqrt(v / (1 - b2 ** e)) + eps)
    return p, np.array(hist)
