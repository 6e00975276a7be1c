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

KIND_NL, KIND_NL_IF, KIND_BRAGG_AD, KIND_DOUBLE_BRAGG_AD, KIND_NL_IF_2, KIND_BRAGG_DS_AD = 0, 1, 2, 3, 4, 5
KIND_NUMERICAL_BRAGG, KIND_NUMERICAL_RAMAN = 6, 7


def gaussian_pulse(tc: float, two_sigma2: float):
    """F(t) for AMP_T = exp(-(t-tc)*(t-tc)/two_sigma2), evaluated in the same
    operation order as the expression parser: ((-(t-tc))*(t-tc))/two_sigma2."""

    def F(t: float) -> float:
        return math.exp((-(t - tc)) * (t - tc) / two_sigma2)

    return F


def laser_kwargs(p: dict, species: int = 1) -> dict:
    """Laser members of CRT_Base_IF (or, species 2, the *_2 members of
    CRT_Base_IF_2: Beta_2, Amp_2, laser_k_2, laser_dk_2, laser_domh_2)."""
    dim = p["dim"]
    sfx = "" if species == 1 else "_2"
    beta = list(p.get("Beta" + sfx, [0.0] * dim)) + [0.0] * (3 - dim)
    return dict(
        beta=beta,
        DeltaL=(list(p.get("Delta_L", [0.0, 0.0])) + [0.0] * 4)[:4],
        Amp=p.get("Amp_1" if species == 1 else "Amp_2", [0.0, 0.0]),
        laser_k=[p.get("laser_k" + sfx, 0.0), 0.0],
        laser_dk=[p.get("laser_dk" + sfx, 0.0), 0.0],
        laser_domh=[p.get("laser_domh" + sfx, 0.0), 0.0],
        phase=[0.0, 0.0],
        chirp_rate=[0.0, 0.0],
        chirp=p.get("chirp", 0.0) if species == 1 else 0.0,
    )


def run_rt(engine, p: dict, psi0, V=None, make_laser=None, on_block=None):
    """Run the sequences of program description ``p`` on ``engine``.

    p keys: dim, ncomp, header_dt (dt stored in the input file), algo_dt
    (ALGORITHM/DT), Alpha_1, gs (flat ncomp^2), sequence = list of dicts
    {name, dt, Nk, duration}, optional AMP_T pulse {tc, two_sigma2}, program
    ('rt_solver', 'bragg', 'double_bragg', 'bragg_ds' or 'raman'; bragg_ds adds
    Alpha_2 and the *_2 laser keys; sequence tags freeprop, bragg_ad and the
    numerical bragg / raman).  Returns the list of (t, [psi per comp]) after every
    block, and the Rabi sums per block of the interferometry programs (both
    species side by side for bragg_ds).
    """
    ncomp = p["ncomp"]
    two_species = p["program"] == "bragg_ds"
    for c in range(ncomp):
        engine.set_psi(c, psi0[c])
    engine.set_dt(p["header_dt"])  # Init() inside the constructor, alpha still zero
    for c in range(ncomp):
        # CRT_Base_2: Alpha_2 for the second species (components ncomp/2 ..)
        engine.set_alpha(c, p["Alpha_2"] if two_species and 2 * c >= ncomp else p["Alpha_1"])
    engine.set_gs(np.asarray(p["gs"], dtype=np.float64))
    cur_dt = p["algo_dt"]
    if V is not None:
        engine.set_potential(0, V)
    laser = make_laser(**laser_kwargs(p)) if make_laser is not None else None
    laser2 = make_laser(**laser_kwargs(p, 2)) if make_laser is not None and two_species else None
    F = gaussian_pulse(p["AMP_T"]["tc"], p["AMP_T"]["two_sigma2"]) if p.get("AMP_T") else None
    outputs, rabi = [], []
    is_if = p["program"] in ("bragg", "double_bragg", "bragg_ds", "raman")
    for seq in p["sequence"]:
        durs = seq["duration"] if isinstance(seq["duration"], list) else [seq["duration"]]
        subN = int(max(durs) / seq["dt"])
        nk = seq["Nk"]
        na = subN // nk
        if cur_dt != seq["dt"]:
            engine.set_dt(seq["dt"])
            cur_dt = seq["dt"]
        if seq["name"] == "bragg_ad":
            kind = {"double_bragg": KIND_DOUBLE_BRAGG_AD, "bragg_ds": KIND_BRAGG_DS_AD}.get(p["program"],
                                                                                         KIND_BRAGG_AD)
        elif seq["name"] == "raman":
            kind = KIND_NUMERICAL_RAMAN
        elif seq["name"] == "bragg":
            kind = KIND_NUMERICAL_BRAGG
        elif two_species:
            kind = KIND_NL_IF_2
        elif is_if:
            kind = KIND_NL_IF
        else:
            kind = KIND_NL
        if two_species and laser2 is not None:
            # seq.time = Get_t() at the start of the sequence; pulse windows
            # from the durations (bragg_ds.cpp:117-127 reads two)
            engine.set_species2(laser2, engine.t, (durs + durs)[:2])
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
                r = engine.rabi_integrals(p["rabi_k0"], p["rabi_threshold"])
                if two_species:  # species 2 on component ncomp/2
                    r = np.concatenate([r, engine.rabi_integrals(p["rabi_k0_2"], p["rabi_threshold"], ncomp // 2)])
                rabi.append(r)
            if on_block is not None:
                on_block(engine)
    return outputs, rabi
