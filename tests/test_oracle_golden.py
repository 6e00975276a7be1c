"""The oracle restatement reproduces the reference programs bit for bit.

The golden fixtures were produced by ATUS-2's own rt_solver / bragg /
double_bragg / bragg_ds / raman / sobmin
compiled from the reference sources (tests/golden/make_golden.py); the
restatement (oracle/atus_oracle.c) replays the same XML programs here.
"""
import numpy as np
import pytest

from golden_io import BRAGG_CASES, BRAGGDS_CASES, DBRAGG_CASES, NUM_CASES, RT_CASES, SOB_CASES, load, sob_inputs
from oracle.oracle import Laser, Oracle
from replay import run_rt


@pytest.mark.parametrize("name", RT_CASES + BRAGG_CASES + DBRAGG_CASES + BRAGGDS_CASES + NUM_CASES)
def test_realtime_bit_exact(name):
    g = load(name)
    p = g["params"]
    o = Oracle(g["header"], p["ncomp"])
    V = g["V"] if "V" in g else None
    outs, rabi = run_rt(o, p, g["psi0"], V=V, make_laser=Laser.make)
    assert len(outs) == len(g["t"])
    for (t, psi), t_ref, psi_ref in zip(outs, g["t"], g["psi"]):
        assert t == t_ref
        for c in range(p["ncomp"]):
            np.testing.assert_array_equal(psi[c], psi_ref[c])
    if p["program"] in ("bragg", "double_bragg", "bragg_ds", "raman"):
        # Rabi_<seq>_<chirp>.txt holds 6 significant digits
        np.testing.assert_allclose(np.array(rabi), g["rabi"], rtol=5e-6, atol=1e-12)


def test_tables_built_before_alpha_is_read():
    """With ALGORITHM/DT equal to the sequence dt the reference never rebuilds
    its kinetic tables after the constructor, which built them with alpha = 0
    (include/CRT_Base.h:147-173, 757-758): the kinetic step is the identity."""
    a, b = load("rt1d"), load("rt1d_tables_at_ctor")
    assert not np.array_equal(a["psi"], b["psi"])
    g = b
    p = dict(g["params"])
    o = Oracle(g["header"], 1)
    outs, _ = run_rt(o, p, g["psi0"], V=g["V"])
    np.testing.assert_array_equal(outs[-1][1][0], g["psi"][-1][0])


@pytest.mark.parametrize("name", SOB_CASES)
def test_sobmin_bit_exact(name):
    g = load(name)
    p = g["params"]
    o = Oracle(g["header"], 1)
    guess, V = sob_inputs(p, g["header"])
    o.set_psi(0, guess)
    o.set_potential(0, V)
    o.set_gs([p["g"] * np.sqrt(p["Nparticles"]) * np.sqrt(p["Nparticles"])])
    o.sob_init([p["alpha"]], p["stepsize"])
    it, res = o.sob_run(p["epsilon"], 100000)
    assert it == int(g["iterations"])
    assert res <= p["epsilon"]
    np.testing.assert_allclose(res, g["res"][-1], rtol=1e-5)
    final = o.psi(0) * np.sqrt(p["Nparticles"])
    np.testing.assert_array_equal(final, g["psi"])
