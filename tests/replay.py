"""Replays an ATUS-2 XML program on a solver engine.

``run_rt`` follows ``CRT_Base::run_sequence`` (include/CRT_Base.h:684-841) and
``CRT_Base_IF::run_sequence`` (include/CRT_Base_IF.h:638-946) for the
sequences the tests use (freeprop / bragg_ad blocks, outputs every Nk steps,
Rabi sums), including the constructor order of CRT_Base (include/CRT_Base.h:
138-175): the kinetic tables are first built before Alpha_1 is read and are
rebuilt only when a sequence's dt differs from the current header dt.

An engine is anything with the ``Oracle`` method set (oracle/oracle.py); the
GPU solver (atus2_b200.Solver) has the same methods, so the same replay checks
both.
"""
from __future__ import annotations

import math

import numpy as np

KIND_NL, KIND_NL_IF, KIND_BRAGG_AD, KIND_DOUBLE_BRAGG_AD = 0, 1, 2, 3


def gaussian_pulse(tc: float, two_sigma2: float):
    """F(t) for AMP_T = exp(-(t-tc)*(t-tc)/two_sigma2), evaluated in the same
    operation order as the expression parser: ((-(t-tc))*(t-tc))/two_sigma2."""

    def F(t: float) -> float:
        return math.exp((-(t - tc)) * (t - tc) / two_sigma2)

    return F


def laser_kwargs(p: dict) -> dict:
    dim = p["dim"]
    beta = list(p.get("Beta", [0.0] * dim)) + [0.0] * (3 - dim)
    return dict(
        beta=beta,
        DeltaL=(list(p.get("Delta_L", [0.0, 0.0])) + [0.0] * 4)[:4],
        Amp=p.get("Amp_1", [0.0, 0.0]),
        laser_k=[p.get("laser_k", 0.0), 0.0],
        laser_dk=[p.get("laser_dk", 0.0), 0.0],
        laser_domh=[p.get("laser_domh", 0.0), 0.0],
        phase=[0.0, 0.0],
        chirp_rate=[0.0, 0.0],
        chirp=p.get("chirp", 0.0),
    )


def run_rt(engine, p: dict, psi0, V=None, make_laser=None, on_block=None):
    """Run the sequences of program description ``p`` on ``engine``.

    p keys: dim, ncomp, header_dt (dt stored in the input file), algo_dt
    (ALGORITHM/DT), Alpha_1, gs (flat ncomp^2), sequence = list of dicts
    {name, dt, Nk, duration}, optional AMP_T pulse {tc, two_sigma2}, program
    ('rt_solver', 'bragg' or 'double_bragg').  Returns the list of (t, [psi per comp]) after
    every block, and the Rabi sums per block when the program is bragg.
    """
    ncomp = p["ncomp"]
    for c in range(ncomp):
        engine.set_psi(c, psi0[c])
    engine.set_dt(p["header_dt"])  # Init() inside the constructor, alpha still zero
    for c in range(ncomp):
        engine.set_alpha(c, p["Alpha_1"])
    engine.set_gs(np.asarray(p["gs"], dtype=np.float64))
    cur_dt = p["algo_dt"]
    if V is not None:
        engine.set_potential(0, V)
    laser = make_laser(**laser_kwargs(p)) if make_laser is not None else None
    F = gaussian_pulse(p["AMP_T"]["tc"], p["AMP_T"]["two_sigma2"]) if p.get("AMP_T") else None
    outputs, rabi = [], []
    is_if = p["program"] in ("bragg", "double_bragg")
    for seq in p["sequence"]:
        subN = int(seq["duration"] / seq["dt"])
        nk = seq["Nk"]
        na = subN // nk
        if cur_dt != seq["dt"]:
            engine.set_dt(seq["dt"])
            cur_dt = seq["dt"]
        if seq["name"] == "bragg_ad":
            kind = KIND_DOUBLE_BRAGG_AD if p["program"] == "double_bragg" else KIND_BRAGG_AD
        elif is_if:
            kind = KIND_NL_IF
        else:
            kind = KIND_NL
        for _ in range(na):
            Fv = None
            if kind in (KIND_BRAGG_AD, KIND_DOUBLE_BRAGG_AD):
                t = engine.t + 0.5 * seq["dt"]
                Fv = []
                for j in range(nk):
                    Fv.append(F(t + 0.5 * seq["dt"]) if F else 1.0)
                    t += seq["dt"]
                Fv = np.array(Fv)
            engine.block(nk, kind, laser, Fv)
            outputs.append((engine.t, [np.array(engine.psi(c)) for c in range(ncomp)]))
            if is_if and seq.get("rabi", False):
                rabi.append(engine.rabi_integrals(p["rabi_k0"], p["rabi_threshold"]))
            if on_block is not None:
                on_block(engine)
    return outputs, rabi
