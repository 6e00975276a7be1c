"""The 1D split step written with numpy's FFT (pocketfft), for calibration.

Same formulas and operation order as the reference's CRT_Base for one
component (include/CRT_Base.h:252-441): kinetic table (cos, sin) of
(-dt)*((k alpha) k), forward transform scaled by dx/sqrt(2 pi), table
multiply, inverse transform scaled by dk/sqrt(2 pi), potential phase.  Only
the FFT differs from the oracle.  Running both shows how far two correct FP64
FFT implementations drift apart on a long nonlinear run -- the yardstick for
the GPU's FFT.
"""
import math

import numpy as np


def run_blocks(x, k, psi, V, g, alpha, dt, nk, nblocks, dx, dk):
    phi = (-dt) * ((k * alpha) * k)
    Th = np.cos(0.5 * phi) + 1j * np.sin(0.5 * phi)
    Tf = np.cos(phi) + 1j * np.sin(phi)
    sf = dx / math.sqrt(2 * math.pi)
    sb = dk / math.sqrt(2 * math.pi)

    def kin(p, T):
        q = np.fft.fft(p) * sf * T
        return np.fft.ifft(q) * len(q) * sb

    def nl(p):
        ph = (V + g * (p.real * p.real + p.imag * p.imag)) * (-dt)
        return p * (np.cos(ph) + 1j * np.sin(ph))

    out = []
    for _ in range(nblocks):
        psi = kin(psi, Th)
        for _j in range(nk - 1):
            psi = kin(nl(psi), Tf)
        psi = kin(nl(psi), Th)
        out.append(psi.copy())
    return out
