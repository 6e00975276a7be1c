"""Loads the golden fixtures written by tests/golden/make_golden.py."""
import json
import math
import os

import numpy as np

from atus2_b200 import binfmt

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

RT_CASES = ["rt1d", "rt1d_tables_at_ctor", "rt2d_slit", "rt3d"]
BRAGG_CASES = ["bragg1d", "bragg2d", "bragg3d"]
DBRAGG_CASES = ["dbragg1d", "dbragg2d", "dbragg3d"]
BRAGGDS_CASES = ["braggds1d", "braggds2d", "braggds3d"]
NUM_CASES = ["raman1d", "raman2d", "raman3d", "nbragg2d"]
SOB_CASES = ["sob1d", "sob2d", "sob3d"]


def load(name):
    z = np.load(os.path.join(HERE, name + ".npz"))
    d = {k: z[k] for k in z.files}
    d["header"] = np.frombuffer(d["header"].tobytes(), dtype=binfmt.HEADER_DTYPE)[0].copy()
    d["params"] = json.loads(str(d["params"]))
    return d


def libm(f, arr):
    flat = np.asarray(arr, dtype=np.float64).ravel()
    return np.array([f(float(v)) for v in flat]).reshape(np.shape(arr))


def sob_inputs(p, header):
    """Guess and potential of a sobmin golden case, evaluated in the same
    operation order as the expression parser evaluates GUESS_xD / POTENTIAL_xD."""
    dim = p["dim"]
    X = np.meshgrid(*[binfmt.x_coords(header, a) for a in range(dim)], indexing="ij")
    if dim == 1:
        (x,) = X
        guess = libm(math.exp, (-0.5 * x) * x)
        V = 0.5 * x * x
    elif dim == 2:
        x, y = X
        guess = libm(math.exp, -0.5 * (x * x + y * y))
        V = 0.5 * (x * x + 4 * y * y)
    else:
        x, y, z = X
        guess = libm(math.exp, -0.5 * (x * x + y * y + z * z))
        V = 0.5 * (x * x + y * y + z * z)
    return guess.astype(np.complex128), V
