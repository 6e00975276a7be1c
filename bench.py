#!/usr/bin/env python
"""Benchmark of the split-step Gross-Pitaevskii path on B200.

Workload (the 3D two-component Bragg configuration): 256^3 grid on
[-32,32)^3, two components, g11 = g12 = g21 = g22 = 100, alpha = 1/2,
coupling Omega(t) cos(2 k_L x - delta t)/2 with k_L = 4 (laser_k = 8),
delta = 16 (laser_domh), Gaussian pulse of peak 8 (Amp = 4) and sigma_t = 0.5
centred at t = 2.5, state 1 a Thomas-Fermi profile (omega = 1) normalised on
the grid, state 2 empty, dt = 1e-3.  The timed window sits on the pulse
(header time starts at 2.4).  Synthetic inputs, seeded.

A step is one Strang step of the bragg_ad sequence over the whole grid; the
metric is grid-point steps per second (grid points x steps / time).  value:
fields resident in HBM, K steps as one run_sequence block (the fused GPU
path), timed with CUDA events on the launching stream.  e2e: the same metric
through the C ABI with host buffers -- every step of the e2e loop is one
output block of 100 Strang steps framed by the host->device upload and the
device->host download of both components (pinned host memory); the steps
alternate between two contexts driven by two host threads, so one context's
copies overlap the other's Strang steps.

Variants in the same JSON line: the mixed-precision form of the same
workload (complex64 fields, FP64 phase arguments) with its error against the
FP64 path after 10^4 steps (5000 pulse + 5000 free steps); the 1D rt_solver
workload (N = 4096, 20000 steps) and the 2D double slit (2048^2, FP64 and
mixed, 10^4-step accuracy); the batched Bragg sweep; sobmin time to residual
1e-10 with and without the learned guess.  Each carries the reference
program's rate on this host's cores where one is timed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl atus|reference]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 256
L = 64.0
G = 100.0
DT = 1e-3
T0 = 2.4
PULSE_TC, PULSE_SIGMA = 2.5, 0.5
E2E_NK = 100
METRIC = "grid-pt-steps/s (3D 256^3 two-component Bragg split-step, FP64)"
UNIT = "grid-pt-steps/s"


def pulse(t: float) -> float:
    return math.exp((-(t - PULSE_TC)) * (t - PULSE_TC) / (2 * PULSE_SIGMA * PULSE_SIGMA))


def pulse_train(t0: float, nk: int):
    """Pulse amplitudes of the nk potential steps of a block starting at t0,
    with the reference's header-time additions (include/CRT_Base.h:361,391)."""
    t = t0 + 0.5 * DT
    out = []
    for _ in range(nk):
        out.append(pulse(t + 0.5 * DT))
        t += DT
    return np.array(out)


def header(n=N):
    from atus2_b200 import binfmt

    return binfmt.make_header(3, [n, n, n], [-L / 2] * 3, [L / 2] * 3, t=T0, dt=DT)


def initial_state(h):
    from atus2_b200 import binfmt

    n = int(h["nDimX"])
    x = binfmt.x_coords(h, 0)
    r2 = x[:, None, None] ** 2 + x[None, :, None] ** 2 + x[None, None, :] ** 2
    mu = 10.0
    psi1 = np.sqrt(np.maximum(0.0, (mu - 0.5 * r2) / G)).astype(np.complex128)
    psi1 /= math.sqrt(float(h["dx"] * h["dy"] * h["dz"]) * float(np.sum(np.abs(psi1) ** 2)))
    psi2 = np.zeros((n, n, n), dtype=np.complex128)
    return psi1, psi2


def laser_kw():
    return dict(Amp=[4.0, 4.0], laser_k=[8.0, 0.0], laser_domh=[16.0, 0.0])


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ helpers
def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, 0, None
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    backend = "nccl" if torch.cuda.is_available() else "gloo"
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=timedelta(seconds=300))
    return rank, ws, local, dist


def max_over_ranks(dist, v: float) -> float:
    if dist is None:
        return v
    import torch

    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist):
    if dist is not None:
        dist.barrier()


def whole_job_rate(ws: int, units_per_rank: float, ms_max: float) -> float:
    """Replicas: every rank processes the same units; the job rate is all
    ranks' units over the slowest rank's device time."""
    return ws * units_per_rank / (ms_max * 1e-3)


# ------------------------------------------------------------------ atus arm
def run_gpu(prec, steps, warmup, stream):
    """Returns (solver, ms for `steps` Strang steps, launches) on a resident state."""
    import torch

    from atus2_b200 import STEP_BRAGG_AD, Laser, Solver

    h = header()
    psi1, psi2 = initial_state(h)
    s = Solver(h, 2, prec)
    s.set_stream(stream.cuda_stream)
    s.set_psi(0, psi1)
    s.set_psi(1, psi2)
    for c in range(2):
        s.set_alpha(c, [0.5, 0.5, 0.5])
    s.set_gs([G] * 4)
    s.set_dt(DT)
    s.set_laser(Laser.make(**laser_kw()))
    for _ in range(warmup):
        s.block(1, STEP_BRAGG_AD, None, pulse_train(s.t, 1))
    F = pulse_train(s.t, steps)
    torch.cuda.synchronize()
    n0 = s.launches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.block(steps, STEP_BRAGG_AD, None, F)
    e1.record(stream)
    torch.cuda.synchronize()
    return s, e0.elapsed_time(e1), s.launches - n0, h


def run_e2e(steps, stream):
    """`steps` cycles of upload (both components, pinned host memory) ->
    E2E_NK Strang steps -> download, through the C ABI, on two contexts
    ("lanes") driven by two host threads: cycle i runs on lane i % 2, so one
    lane's copies overlap the other lane's steps (independent states, as in
    a scan).  Wall time between two device synchronisations."""
    import torch

    from atus2_b200 import PREC_FP64, STEP_BRAGG_AD, Laser, Solver

    h = header()
    psi1, psi2 = initial_state(h)
    npts = N ** 3
    lanes = []
    for _ in range(2):
        host = [torch.empty(2 * npts, dtype=torch.float64, pin_memory=True) for _ in range(2)]
        host[0].numpy()[:] = psi1.view(np.float64).ravel()
        host[1].numpy()[:] = psi2.view(np.float64).ravel()
        s = Solver(h, 2, PREC_FP64)
        st = torch.cuda.Stream()
        s.set_stream(st.cuda_stream)
        for c in range(2):
            s.set_alpha(c, [0.5, 0.5, 0.5])
        s.set_gs([G] * 4)
        s.set_dt(DT)
        s.set_laser(Laser.make(**laser_kw()))
        lanes.append((s, host, st))

    def cycle(s, host, nk):
        for c in range(2):
            s.upload_from(c, host[c].data_ptr())
        s.block(nk, STEP_BRAGG_AD, None, pulse_train(s.t, nk))
        for c in range(2):
            s.download_to(c, host[c].data_ptr())

    for s, host, _ in lanes:  # one untimed round trip per lane
        cycle(s, host, 2)
    torch.cuda.synchronize()

    def run_lane(k):
        s, host, _ = lanes[k]
        for _ in range(k, steps, 2):
            cycle(s, host, E2E_NK)

    t0 = time.perf_counter()
    threads = [threading.Thread(target=run_lane, args=(k,)) for k in range(2)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1e3
    for s, _, _ in lanes:
        s.close()
    return ms, 2 * 16 * npts, 2 * 16 * npts


# ------------------------------------------------------------------ accuracy at full length
ACC_PULSE_STEPS, ACC_FREE_STEPS, ACC_NK = 5000, 5000, 1000


def _norm(s, ncomp):
    return sum(s.particle_number(c) for c in range(ncomp))


def run_accuracy3(stream):
    """The 256^3 Bragg workload at full length from t = 0: 5000 bragg_ad steps
    (pulse centred at 2.5, sigma 0.5) then 5000 freeprop steps, in blocks of
    1000, in FP64 and in mixed precision.  The FP64 GPU path is the yardstick
    (it matches the oracle to 1e-11 at this grid in the tests; the oracle
    itself would need hours for 10^4 steps).  Returns the relative L2 error of
    the mixed state per component and in total, the norm drift of both forms
    and the Rabi populations."""
    import torch

    from atus2_b200 import PREC_FP64, PREC_MIXED, STEP_BRAGG_AD, STEP_NL_IF, Laser, Solver

    h = header()
    h["t"] = 0.0
    psi1, psi2 = initial_state(h)
    res = {}
    final = {}
    for name, prec in (("fp64", PREC_FP64), ("mixed", PREC_MIXED)):
        s = Solver(h, 2, prec)
        s.set_stream(stream.cuda_stream)
        s.set_psi(0, psi1)
        s.set_psi(1, psi2)
        for c in range(2):
            s.set_alpha(c, [0.5, 0.5, 0.5])
        s.set_gs([G] * 4)
        s.set_dt(DT)
        s.set_laser(Laser.make(**laser_kw()))
        n0 = _norm(s, 2)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(ACC_PULSE_STEPS // ACC_NK):
            s.block(ACC_NK, STEP_BRAGG_AD, None, pulse_train(s.t, ACC_NK))
        pops_pulse = [s.particle_number(c) for c in range(2)]
        for _ in range(ACC_FREE_STEPS // ACC_NK):
            s.block(ACC_NK, STEP_NL_IF)
        s.synchronize()
        wall = time.perf_counter() - t0
        n1 = _norm(s, 2)
        res[name] = {"norm_drift": (n1 - n0) / n0, "populations_after_pulse": pops_pulse,
                     "populations_end": [s.particle_number(c) for c in range(2)], "wall_s": wall}
        final[name] = [s.psi(c) for c in range(2)]
        s.close()
    ref, got = final["fp64"], final["mixed"]
    err = [float(np.linalg.norm(g - r) / np.linalg.norm(r)) for g, r in zip(got, ref)]
    tot = float(math.sqrt(sum(np.linalg.norm(g - r) ** 2 for g, r in zip(got, ref)) /
                          sum(np.linalg.norm(r) ** 2 for r in ref)))
    res["mixed"]["rel_l2_vs_fp64"] = {"component_1": err[0], "component_2": err[1], "state": tot}
    res["steps"] = ACC_PULSE_STEPS + ACC_FREE_STEPS
    res["sequence"] = (f"{ACC_PULSE_STEPS} bragg_ad + {ACC_FREE_STEPS} freeprop steps from t = 0, blocks of {ACC_NK}, "
                       "dt = 1e-3")
    res["bar"] = "relative L2 <= 1e-5 against FP64 after 10^4 steps"
    return res


# ------------------------------------------------------------------ config 1: 1D rt_solver
C1_N, C1_NK, C1_BLOCKS = 4096, 1000, 20


def config1_inputs():
    """N = 4096 on [-100,100), V = x^2/2, psi = exp(-(x-5)^2/2) e^{2ix} plus
    complex noise of amplitude 1e-6 (seed 0), normalised; g = 10, dt = 1e-3."""
    from atus2_b200 import binfmt

    h = binfmt.make_header(1, [C1_N], [-100.0], [100.0], dt=DT)
    x = binfmt.x_coords(h, 0)
    rng = np.random.default_rng(0)
    psi = np.exp(-0.5 * (x - 5) ** 2) * np.exp(2j * x) + 1e-6 * (rng.standard_normal(C1_N) +
                                                              1j * rng.standard_normal(C1_N))
    psi /= math.sqrt(float(h["dx"]) * float(np.sum(np.abs(psi) ** 2)))
    return h, psi, 0.5 * x * x


def run_config1(stream, with_cpu):
    """Config 1 at full length: 20 blocks of 1000 Strang steps of the 1D
    rt_solver workload, FP64, one CTA holding the field in shared memory."""
    import torch

    from atus2_b200 import PREC_FP64, STEP_NL, Solver

    h, psi, V = config1_inputs()
    s = Solver(h, 1, PREC_FP64)
    s.set_stream(stream.cuda_stream)
    s.set_psi(0, psi)
    s.set_alpha(0, [0.5])
    s.set_gs([10.0])
    s.set_potential(0, V)
    s.set_dt(DT)
    s.block(C1_NK, STEP_NL)  # warm-up block (state advances; timing only)
    s.set_psi(0, psi)
    s.t = 0.0
    n0 = s.particle_number(0)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = s.launches
    e0.record(stream)
    for _ in range(C1_BLOCKS):
        s.block(C1_NK, STEP_NL)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    steps = C1_NK * C1_BLOCKS
    out = {
        "metric": "grid-pt-steps/s (1D rt_solver, N=4096, FP64)",
        "value": C1_N * steps / (ms * 1e-3),
        "unit": UNIT,
        "ms": ms,
        "steps": steps,
        "us_per_step": ms * 1e3 / steps,
        "gpu_launches": s.launches - l0,
        "norm_drift": (s.particle_number(0) - n0) / n0,
        "dtype": "f64",
        "bound": "latency / FP64 issue of one SM: the 64 KB field stays in one CTA's shared memory for a "
                 "whole block, so HBM is not on the path (72 B/pt-step model: "
                 f"{72.0 * C1_N * steps / (ms * 1e-3) / 1e9:.1f} GB/s equivalent)",
    }
    s.close()
    if with_cpu and _ref_prog("rt_solver"):
        from atus2_b200 import binfmt

        def inputs(tmp):
            binfmt.write_bin(os.path.join(tmp, "inp_1.bin"), h, psi)

        def xml(ns):
            return f"""<SIMULATION>
  <DIM>1</DIM><FILENAME>inp_1.bin</FILENAME><POTENTIAL_1D>0.5*x*x</POTENTIAL_1D>
  <CONSTANTS><unused>0</unused></CONSTANTS>
  <VCONSTANTS><Alpha_1>0.5</Alpha_1><GS_1>10</GS_1></VCONSTANTS>
  <ALGORITHM><DT>0.001</DT></ALGORITHM>
  <SEQUENCE><freeprop dt="0.001" Nk="{ns}" output_freq="none" pn_freq="none">{ns * DT!r}</freeprop></SEQUENCE>
</SIMULATION>"""

        r = time_ref_program(_ref_prog("rt_solver"), inputs, xml, 1000, 5000, repeats=3)
        if r:
            out["cpu_reference"] = {"value": C1_N / r["per_step_s"], "unit": UNIT, "cores": r["cores"],
                                    "kind": "reference", "sample": f"ATUS-2 rt_solver (oracle/_ref, shim FFT), "
                                    f"{r['runs']} freeprop steps, difference of medians", "wall_s": r["wall_s"]}
    return out


# ------------------------------------------------------------------ config 2: 2D double slit
C2_N, C2_L, C2_DT, C2_G = 2048, 128.0, 5e-4, 1.0
C2_V_EXPR = "200*rect(x,-0.5,0.5)*(1-rect(y,-5,-3)-rect(y,3,5))"


def config2_inputs():
    """2048^2 on [-64,64)^2: V = 200 on |x| < 0.5 except the slits |y -+ 4| < 1,
    packet exp(-((x+20)^2 + y^2)/32) e^{8ix} normalised, g = 1, dt = 5e-4."""
    from atus2_b200 import binfmt

    h = binfmt.make_header(2, [C2_N, C2_N], [-C2_L / 2] * 2, [C2_L / 2] * 2, dt=C2_DT)
    x = binfmt.x_coords(h, 0)[:, None]
    y = binfmt.x_coords(h, 1)[None, :]
    V = np.where((np.abs(x) < 0.5) & ~((np.abs(y - 4) < 1) | (np.abs(y + 4) < 1)), 200.0, 0.0)
    psi = np.exp(-((x + 20) ** 2 + y ** 2) / 32.0) * np.exp(8j * x)
    psi /= math.sqrt(float(h["dx"] * h["dy"]) * float(np.sum(np.abs(psi) ** 2)))
    return h, psi, V


def _c2_solver(prec, stream, h, psi, V):
    from atus2_b200 import Solver

    s = Solver(h, 1, prec)
    s.set_stream(stream.cuda_stream)
    s.set_psi(0, psi)
    s.set_alpha(0, [0.5, 0.5])
    s.set_gs([C2_G])
    s.set_potential(0, V)
    s.set_dt(C2_DT)
    return s


def run_config2(stream, steps, warmup, peak, peak_kind, with_cpu, accuracy=True):
    """Config 2: throughput of `steps` Strang steps as one block (fields
    resident), FP64 and mixed, with the per-pass roofline (72 B/pt-step FP64,
    40 B mixed: 2 half steps x read+write of the field + the FP64 potential);
    then 10^4 steps (10 blocks of 1000) of both forms for the mixed form's
    error and the norm drift."""
    import torch

    from atus2_b200 import PREC_FP64, PREC_MIXED, STEP_NL

    h, psi, V = config2_inputs()
    npts = C2_N * C2_N
    out = {"metric": "grid-pt-steps/s (2D double slit, 2048^2)", "unit": UNIT,
           "l2": "field 64 MB (FP64) + potential 32 MB: below the 126 MB L2 in part; DRAM bytes from ncu"}
    for name, prec, model in (("fp64", PREC_FP64, 72.0), ("mixed", PREC_MIXED, 40.0)):
        s = _c2_solver(prec, stream, h, psi, V)
        s.block(warmup, STEP_NL)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = s.launches
        e0.record(stream)
        s.block(steps, STEP_NL)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        rate = npts * steps / (ms * 1e-3)
        prof = s.profile_passes(STEP_NL, reps=5)
        names = ["x pass (FFT_x, kinetic, IFFT_x)", "y pass (IFFT_y, potential, FFT_y)"]
        out[name] = {
            "value": rate, "ms_per_step": ms / steps, "gpu_launches": s.launches - l0,
            "model_bytes_per_pt_step": model,
            "roofline": {"bound": "hbm", "achieved": model * rate / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": model * rate / 1e9 / peak, "peak_source": peak_kind,
                         "passes": [{"kernel": names[q] if q < len(names) else f"pass {q}", "ms": p[0],
                                     "bytes": p[2], "GBps": p[2] / (p[0] * 1e-3) / 1e9} for q, p in enumerate(prof)]},
        }
        s.close()
    out["mixed"]["speedup_vs_fp64"] = out["fp64"]["ms_per_step"] / out["mixed"]["ms_per_step"]
    out["value"] = out["fp64"]["value"]
    if accuracy:
        final = {}
        for name, prec in (("fp64", PREC_FP64), ("mixed", PREC_MIXED)):
            s = _c2_solver(prec, stream, h, psi, V)
            n0 = s.particle_number(0)
            for _ in range(10):
                s.block(1000, STEP_NL)
            out[name]["norm_drift_10k"] = (s.particle_number(0) - n0) / n0
            final[name] = s.psi(0)
            s.close()
        out["mixed"]["rel_l2_vs_fp64_10k"] = float(np.linalg.norm(final["mixed"] - final["fp64"]) /
                                                   np.linalg.norm(final["fp64"]))
        out["accuracy_steps"] = 10000
    if with_cpu and _ref_prog("rt_solver"):
        from atus2_b200 import binfmt

        def inputs(tmp):
            binfmt.write_bin(os.path.join(tmp, "inp_1.bin"), h, psi)

        def xml(ns):
            return f"""<SIMULATION>
  <DIM>2</DIM><FILENAME>inp_1.bin</FILENAME><POTENTIAL_2D>{C2_V_EXPR}</POTENTIAL_2D>
  <CONSTANTS><unused>0</unused></CONSTANTS>
  <VCONSTANTS><Alpha_1>0.5,0.5</Alpha_1><GS_1>1</GS_1></VCONSTANTS>
  <ALGORITHM><DT>0.0005</DT></ALGORITHM>
  <SEQUENCE><freeprop dt="0.0005" Nk="{ns}" output_freq="none" pn_freq="none">{ns * C2_DT!r}</freeprop></SEQUENCE>
</SIMULATION>"""

        r = time_ref_program(_ref_prog("rt_solver"), inputs, xml, 2, 8, repeats=3)
        if r:
            out["cpu_reference"] = {"value": npts / r["per_step_s"], "unit": UNIT, "cores": r["cores"],
                                    "kind": "reference", "sample": f"ATUS-2 rt_solver (oracle/_ref, shim FFT), "
                                    f"{r['runs']} freeprop steps, difference of medians", "wall_s": r["wall_s"]}
    return out


def _ref_prog(name):
    p = os.path.join(ROOT, "oracle", "_ref", name)
    return p if os.path.exists(p) else None


def time_ref_program(prog, make_inputs, xml_for, n_short, n_long, repeats=3, timeout=900):
    """Wall time of the reference program ``prog`` (oracle/_ref, built from
    the ATUS-2 sources with the FFTW-API shim) on all host cores, for runs of
    n_short and n_long Strang steps, each repeated; the per-step cost is the
    difference of the medians over (n_long - n_short), so the set-up (file
    reads, tables, potentials) cancels.  make_inputs(tmp) writes the input
    files, xml_for(nsteps) returns the run's XML."""
    cores = os.cpu_count() or 1
    env = dict(os.environ, MY_NO_OF_THREADS=str(cores), OMP_NUM_THREADS=str(cores))
    times = {n_short: [], n_long: []}
    with tempfile.TemporaryDirectory() as tmp:
        make_inputs(tmp)
        for _ in range(repeats):
            for ns in (n_short, n_long):
                open(os.path.join(tmp, "run.xml"), "w").write(xml_for(ns))
                t0 = time.perf_counter()
                r = subprocess.run([prog, "run.xml"], cwd=tmp, env=env, capture_output=True, text=True,
                                   timeout=timeout)
                times[ns].append(time.perf_counter() - t0)
                if r.returncode != 0:
                    return None
    med_s, med_l = statistics.median(times[n_short]), statistics.median(times[n_long])
    per_step = max((med_l - med_s) / (n_long - n_short), 1e-12)
    # spread: the per-step cost from the fastest and slowest pairing of runs
    lo = max((min(times[n_long]) - max(times[n_short])) / (n_long - n_short), 1e-12)
    hi = max((max(times[n_long]) - min(times[n_short])) / (n_long - n_short), 1e-12)
    return {"per_step_s": per_step, "per_step_range_s": [lo, hi], "cores": cores, "seconds": times,
            "runs": f"{repeats} x ({n_short} and {n_long} steps)", "wall_s": sum(times[n_short]) + sum(times[n_long])}


def bragg_xml(ns, pulse_tc=PULSE_TC, pulse_sigma=PULSE_SIGMA):
    """bragg program input for the 256^3 workload: one bragg_ad block of ns steps."""
    return f"""<SIMULATION>
  <DIM>3</DIM><FILENAME>inp_1.bin</FILENAME><FILENAME_2>inp_2.bin</FILENAME_2>
  <AMP_T>exp(-(t-{pulse_tc!r})*(t-{pulse_tc!r})/{2 * pulse_sigma * pulse_sigma!r})</AMP_T>
  <CONSTANTS><laser_k>8</laser_k><laser_dk>0</laser_dk><laser_domh>16</laser_domh>
    <rabi_threshold>1</rabi_threshold><chirp>0</chirp></CONSTANTS>
  <VCONSTANTS><Amp_1>4,4</Amp_1><Alpha_1>0.5,0.5,0.5</Alpha_1><Delta_L>0,0</Delta_L>
    <GS_1>100,100</GS_1><GS_2>100,100</GS_2><Beta>0,0,0</Beta></VCONSTANTS>
  <ALGORITHM><DT>1</DT></ALGORITHM>
  <SEQUENCE><bragg_ad dt="0.001" Nk="{ns}" output_freq="none" pn_freq="none">{ns * DT!r}</bragg_ad></SEQUENCE>
</SIMULATION>"""


def run_cpu_baseline(n_short=1, n_long=5, repeats=3):
    """The reference bragg program on this host's cores on the 256^3 Bragg
    workload (the same state and pulse as the GPU runs)."""
    prog = _ref_prog("bragg")
    if prog is None:
        return None
    from atus2_b200 import binfmt

    def inputs(tmp):
        h = header()
        psi1, psi2 = initial_state(h)
        binfmt.write_bin(os.path.join(tmp, "inp_1.bin"), h, psi1)
        binfmt.write_bin(os.path.join(tmp, "inp_2.bin"), h, psi2)

    r = time_ref_program(prog, inputs, bragg_xml, n_short, n_long, repeats)
    if r is None:
        return None
    return {
        "value": N ** 3 / r["per_step_s"],
        "value_range": [N ** 3 / r["per_step_range_s"][1], N ** 3 / r["per_step_range_s"][0]],
        "unit": UNIT,
        "cores": r["cores"],
        "kind": "reference",
        "fft": "FFTW-API shim (oracle/fft_cpu.c, FP64 mixed-radix, OpenMP over pencils); FFTW 3.3.8 is not installed",
        "sample": f"ATUS-2 bragg program (oracle/_ref) at 256^3 x 2 components, {r['runs']} bragg_ad steps "
                  f"(Nk = steps), per-step cost = difference of the medians / {n_long - n_short}; "
                  f"MY_NO_OF_THREADS={r['cores']}",
        "seconds": r["seconds"],
        "wall_s": r["wall_s"],
    }


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the
# FP64 256^3 x 2 kernels, each from one ncu capture of that kernel on this
# workload on a B200 (a profiler cannot run inside the timed bench, so the
# capture's figure is carried here).
NCU_TRAFFIC_FP64 = {"pass2_kernel M2_NL (z)": 1.0941e9, "pass2_tma_kernel M2_KIN (x)": 1.0155e9}


def roofline(s, kind, peak, peak_kind, fp64=True):
    prof = s.profile_passes(kind, reps=5)
    # pass names in atus_profile_passes order: x kinetic pass, then the
    # three axis passes of the real-space half step (strided passes take
    # their tiles by TMA unless ATUS_TMA=0)
    sk = "pass2_kernel" if os.environ.get("ATUS_TMA") == "0" else "pass2_tma_kernel"
    names = [f"{sk} M2_KIN (x)", f"{sk} M2_INV (y)", "pass2_kernel M2_NL (z)", f"{sk} M2_FWD (y)"]
    # dominant pass: largest device time per Strang step
    bi = max(range(len(prof)), key=lambda q: prof[q][0] * prof[q][1])
    ms, lps, by = prof[bi]
    achieved = by / (ms * 1e-3) / 1e9
    name = names[bi] if bi < len(names) else f"pass {bi}"
    traffic = NCU_TRAFFIC_FP64.get(name) if fp64 else None
    return {
        "bound": "hbm",
        "achieved": achieved,
        "peak": peak,
        "unit": "GB/s",
        "frac": achieved / peak,
        "peak_source": peak_kind,
        "traffic": traffic,
        "traffic_source": "ncu capture of this kernel at this size (dram__bytes_read.sum + dram__bytes_write.sum)"
                          if traffic else None,
        "kernel": name,
        "algorithmic_bytes_per_launch": by,
        "passes": [{"kernel": names[q] if q < len(names) else f"pass {q}", "ms": p[0], "launches_per_step": p[1],
                    "bytes": p[2], "GBps": p[2] / (p[0] * 1e-3) / 1e9} for q, p in enumerate(prof)],
    }


def atus_arm(args, rank, ws, local, dist):
    import torch

    from atus2_b200 import PREC_FP64, PREC_MIXED, STEP_BRAGG_AD

    torch.cuda.set_device(local)
    # a stream of its own: the library launches on it and the events are recorded on it
    stream = torch.cuda.Stream()
    peak, peak_kind = peaks()
    with ClockSampler(local) as clk:
        barrier(dist)
        s, ms, launches, h = run_gpu(PREC_FP64, args.steps, args.warmup, stream)
        ms = max_over_ranks(dist, ms)
    npts = N ** 3
    value = whole_job_rate(ws, npts * args.steps, ms)
    out = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded Thomas-Fermi state, analytic potential parameters)",
        "config": {
            "workload": "3D two-component Bragg pulse (bragg_ad), 256^3 on [-32,32)^3, g=100, k_L=4, delta=16, "
                        "Omega peak 8, sigma_t 0.5, dt=1e-3",
            "grid": [N, N, N],
            "components": 2,
            "parallelism": f"replicas x{ws} (no inter-GPU exchange)",
            "l2": "fields (2 x 268 MB) larger than the 126 MB L2; no flush needed",
            "block": f"{args.steps} Strang steps as one run_sequence block",
        },
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if rank == 0:
        out["roofline"] = roofline(s, STEP_BRAGG_AD, peak, peak_kind)
    s.close()
    # mixed precision variant (same workload, complex64 fields)
    barrier(dist)
    sm, msm, lm, _ = run_gpu(PREC_MIXED, args.steps, args.warmup, stream)
    msm = max_over_ranks(dist, msm)
    out["variants"] = {"mixed": {"value": whole_job_rate(ws, npts * args.steps, msm), "ms_per_step": msm / args.steps,
                                 "dtype": "c64 fields, f64 phase arguments", "speedup_vs_fp64": ms / msm}}
    if rank == 0:
        out["variants"]["mixed"]["roofline"] = roofline(sm, STEP_BRAGG_AD, peak, peak_kind, fp64=False)
    sm.close()
    # end-to-end through the C ABI with host buffers
    barrier(dist)
    e2e_steps = 2 * max(2, min(args.steps // 40, 3))
    ms_e, bi, bo = run_e2e(e2e_steps, stream)
    ms_e = max_over_ranks(dist, ms_e)
    out["e2e"] = {"value": whole_job_rate(ws, npts * E2E_NK * e2e_steps, ms_e), "unit": UNIT,
                  "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo,
                  "step": f"upload 2 components, {E2E_NK} Strang steps, download 2 components",
                  "pipelining": "two contexts in two host threads, steps alternating between them, so one "
                                "context's host<->device copies overlap the other's Strang steps; wall clock "
                                "between device synchronisations",
                  "steps": e2e_steps}
    if not args.no_accuracy:
        barrier(dist)
        out["variants"]["mixed"]["accuracy_10k"] = run_accuracy3(stream)
    if not args.no_configs:
        barrier(dist)
        cpu = rank == 0 and ws == 1 and not args.no_cpu_baseline
        out["variants"]["config1_1d"] = run_config1(stream, cpu)
        barrier(dist)
        out["variants"]["config2_2d"] = run_config2(stream, args.steps, args.warmup, peak, peak_kind, cpu,
                                                    accuracy=not args.no_accuracy)
    if args.file_output and rank == 0:
        out["variants"]["file_output"] = run_output_overlap()
    if args.phase_scans and rank == 0:
        out["variants"]["phase_scans"] = run_phase_scans()
    if not args.no_batch:
        barrier(dist)
        out["variants"]["batch"] = run_batch()
    if not args.no_sobmin:
        barrier(dist)
        out["variants"]["sobmin"] = run_sobmin(no_cpu=args.no_cpu_baseline or rank != 0)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = run_cpu_baseline()
    barrier(dist)
    if rank == 0:
        print(json.dumps(out))


# ------------------------------------------------------------------ file output during a run
def run_output_overlap(blocks=4, nk=1000, reps=3):
    """ATUS-2's bragg program built against the drop-in headers (host/bin/
    bragg) on the 256^3 workload: `blocks` blocks of `nk` steps with every
    component written after each block (output_freq="each", 537 MB per
    output), against the same run without output, with the files written
    from snapshots by a writer thread (the default) and synchronously
    (ATUS_SYNC_OUTPUT=1).  Median wall time of `reps` runs of each whole
    program, the three kinds interleaved."""
    prog = os.path.join(ROOT, "atus2_b200", "host", "bin", "bragg")
    if not os.path.exists(prog):
        return {"unavailable": "host/bin/bragg is not built (needs the ATUS-2 source tree at build time)"}
    from atus2_b200 import binfmt

    def xml(freq):
        return bragg_xml(nk).replace(f'Nk="{nk}" output_freq="none"', f'Nk="{nk}" output_freq="{freq}"').replace(
            f">{nk * DT!r}</bragg_ad>", f">{blocks * nk * DT!r}</bragg_ad>")

    out = {"grid": [N, N, N], "components": 2, "blocks": blocks, "steps_per_block": nk,
           "bytes_per_output": 2 * 16 * N ** 3}
    with tempfile.TemporaryDirectory() as tmp:
        h = header()
        psi1, psi2 = initial_state(h)
        binfmt.write_bin(os.path.join(tmp, "inp_1.bin"), h, psi1)
        binfmt.write_bin(os.path.join(tmp, "inp_2.bin"), h, psi2)
        runs = {"no_output": ("none", {}), "async_output": ("each", {}), "sync_output": ("each", {"ATUS_SYNC_OUTPUT": "1"})}
        times = {k: [] for k in runs}
        for _ in range(reps):
            for name, (freq, extra) in runs.items():
                open(os.path.join(tmp, "run.xml"), "w").write(xml(freq))
                env = dict(os.environ, **extra)
                t0 = time.perf_counter()
                r = subprocess.run([prog, "run.xml"], cwd=tmp, env=env, capture_output=True, text=True, timeout=600)
                times[name].append(time.perf_counter() - t0)
                if r.returncode != 0:
                    return {"error": f"{name}: rc {r.returncode}: {r.stdout[-500:]} {r.stderr[-500:]}"}
                for fn in os.listdir(tmp):
                    if fn.endswith(".bin") and not fn.startswith("inp_"):
                        os.remove(os.path.join(tmp, fn))
        for name in runs:
            out[name + "_s"] = statistics.median(times[name])
            out[name + "_all_s"] = times[name]
    out["output_cost_async_s"] = out["async_output_s"] - out["no_output_s"]
    out["output_cost_sync_s"] = out["sync_output_s"] - out["no_output_s"]
    return out


def run_phase_scans(reps=5):
    """ATUS-2's bragg program on the drop-in headers with a phase scan
    (no_of_chirps scans of a bragg_ad sequence, chirp_mode 1, Rabi sums every
    block): scans 1..n-1 side by side on cloned contexts (the default)
    against one after another (ATUS_SEQUENTIAL_SCANS=1).  Median wall time
    of `reps` runs of the whole program, the two kinds interleaved."""
    prog = os.path.join(ROOT, "atus2_b200", "host", "bin", "bragg")
    if not os.path.exists(prog):
        return {"unavailable": "host/bin/bragg is not built (needs the ATUS-2 source tree at build time)"}
    from atus2_b200 import binfmt

    cases = [dict(name="1D-4096", dim=1, n=[4096], L=[128.0], scans=16, nk=400, blocks=10),
             dict(name="2D-512", dim=2, n=[512, 512], L=[32.0, 32.0], scans=8, nk=200, blocks=5)]
    out = {}
    for c in cases:
        dim = c["dim"]
        h = binfmt.make_header(dim, c["n"], [-0.5 * L for L in c["L"]], [0.5 * L for L in c["L"]], dt=DT)
        X = np.meshgrid(*[binfmt.x_coords(h, a) for a in range(dim)], indexing="ij")
        r2 = sum(x * x for x in X)
        psi1 = np.sqrt(np.maximum(0.0, 1.0 - r2 / (0.1 * c["L"][0]) ** 2)).astype(np.complex128)
        vec = lambda v: ",".join(repr(float(a)) for a in v)
        xml = f"""<SIMULATION>
  <DIM>{dim}</DIM><FILENAME>inp_1.bin</FILENAME><FILENAME_2>inp_2.bin</FILENAME_2>
  <AMP_T>exp(-(t-0.2)*(t-0.2)/0.005)</AMP_T>
  <CONSTANTS><laser_k>4</laser_k><laser_dk>0</laser_dk><laser_domh>16</laser_domh>
    <rabi_threshold>1</rabi_threshold><chirp>0</chirp></CONSTANTS>
  <VCONSTANTS><Amp_1>4,4</Amp_1><Alpha_1>{vec([0.5] * dim)}</Alpha_1><Delta_L>0,0</Delta_L>
    <GS_1>100,100</GS_1><GS_2>100,100</GS_2><Beta>{vec([0.05] * dim)}</Beta></VCONSTANTS>
  <ALGORITHM><DT>1</DT></ALGORITHM>
  <SEQUENCE><bragg_ad dt="{DT!r}" Nk="{c['nk']}" output_freq="none" pn_freq="none" rabi_output_freq="each"
    no_of_chirps="{c['scans']}" chirp_mode="1" chirp_min="-2" chirp_max="2">{c['blocks'] * c['nk'] * DT!r}</bragg_ad>
  </SEQUENCE>
</SIMULATION>"""
        times = {"side_by_side": [], "sequential": []}
        with tempfile.TemporaryDirectory() as tmp:
            binfmt.write_bin(os.path.join(tmp, "inp_1.bin"), h, psi1)
            binfmt.write_bin(os.path.join(tmp, "inp_2.bin"), h, np.zeros_like(psi1))
            open(os.path.join(tmp, "run.xml"), "w").write(xml)
            for _ in range(reps):
                for kind, extra in (("side_by_side", {}), ("sequential", {"ATUS_SEQUENTIAL_SCANS": "1"})):
                    t0 = time.perf_counter()
                    r = subprocess.run([prog, "run.xml"], cwd=tmp, env=dict(os.environ, **extra), capture_output=True,
                                       text=True, timeout=600)
                    times[kind].append(time.perf_counter() - t0)
                    if r.returncode != 0:
                        return {"error": f"{c['name']} {kind}: rc {r.returncode}: {r.stdout[-500:]} {r.stderr[-500:]}"}
        out[c["name"]] = {"scans": c["scans"], "steps_per_scan": c["blocks"] * c["nk"],
                          "side_by_side_s": statistics.median(times["side_by_side"]),
                          "sequential_s": statistics.median(times["sequential"]), "all_s": times,
                          "min_s": {k: min(v) for k, v in times.items()},
                          "speedup": statistics.median(times["sequential"]) / statistics.median(times["side_by_side"])}
    return out


# ------------------------------------------------------------------ batched sweep
BATCH_COUNT, BATCH_STEPS, BATCH_SEED = 768, 4000, 1


def run_batch(stream_unused=None):
    """The batched Bragg sweep: BATCH_COUNT instances drawn from seed 1
    (atus2_b200.sweep), complex64 fields with FP64 phase arguments, autotuned,
    BATCH_STEPS steps as one graph launch.  Against it: the same instances one
    by one in plain FP64, timed on one representative instance per size class
    over the full BATCH_STEPS in one FP64 context (1D 8192 with two
    components runs as per-step passes, 1D 16384 as four-step transforms),
    which also gives the accuracy of each class after BATCH_STEPS steps."""
    import torch

    from atus2_b200 import PREC_FP64, PREC_MIXED, STEP_BRAGG_AD, Batch, Solver, sweep

    insts = sweep.draw(BATCH_COUNT, BATCH_SEED)
    b = Batch(insts, PREC_MIXED, DT)
    for i, d in enumerate(insts):
        p = sweep.initial_state(d["header"])
        b.set_psi(i, 0, p)
        b.set_psi(i, 1, np.zeros_like(p))
    t_tune = time.perf_counter()
    b.tune(20)
    t_tune = time.perf_counter() - t_tune
    ms = b.run(BATCH_STEPS)
    classes = {}
    for i, d in enumerate(insts):
        h = d["header"]
        key = (int(h["nDims"]), int(h["nDimX"]))
        classes.setdefault(key, []).append(i)
    seq_ms = {}
    errs = {}
    for key, ids in sorted(classes.items()):
        i = ids[0]
        d = insts[i]
        h = d["header"]
        s = Solver(h, 2, PREC_FP64)
        s.set_bragg_stable(True)  # the reference's eigen-form diverges in this sweep's pulse tails
        p = sweep.initial_state(h)
        s.set_psi(0, p)
        s.set_psi(1, np.zeros_like(p))
        for c in range(2):
            s.set_alpha(c, [0.5] * key[0])
        s.set_gs(d["gs"])
        s.set_dt(DT)
        F = sweep.pulse_values(0.0, BATCH_STEPS, *d["pulse"], DT)
        s.synchronize()
        t0 = time.perf_counter()
        s.block(BATCH_STEPS, STEP_BRAGG_AD, d["laser"], F)
        s.synchronize()
        seq_ms[key] = (time.perf_counter() - t0) * 1e3
        ref = np.stack([s.psi(0), s.psi(1)])
        got = np.stack([b.psi(i, 0), b.psi(i, 1)])
        errs[f"{key[0]}D-{key[1]}"] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
        s.close()
    # the reference's own FP64 form on the same instances (what the drop-in
    # computes): its norm after the run, per class
    ref_norms = {}
    for key, ids in sorted(classes.items()):
        if key[0] != 1 or key[1] > 4096:
            continue
        d = insts[ids[0]]
        h = d["header"]
        s = Solver(h, 2, PREC_FP64)
        p = sweep.initial_state(h)
        s.set_psi(0, p)
        s.set_psi(1, np.zeros_like(p))
        for c in range(2):
            s.set_alpha(c, [0.5])
        s.set_gs(d["gs"])
        s.set_dt(DT)
        s.block(BATCH_STEPS, STEP_BRAGG_AD, d["laser"], sweep.pulse_values(0.0, BATCH_STEPS, *d["pulse"], DT))
        ref_norms[f"1D-{key[1]}"] = s.particle_number(0) + s.particle_number(1)
        s.close()
    seq_total = sum(seq_ms[k] * len(v) for k, v in classes.items())
    work = BATCH_COUNT * BATCH_STEPS
    sched = b.schedule()
    b.close()
    return {
        "metric": "instance-steps/s (batched Bragg sweep)",
        "value": work / (ms * 1e-3),
        "unit": "instance-steps/s",
        "ms": ms,
        "instances": BATCH_COUNT,
        "steps": BATCH_STEPS,
        "dtype": "c64 fields, f64 phase arguments",
        "sequential_fp64": {"value": work / (seq_total * 1e-3), "unit": "instance-steps/s",
                            "ms": seq_total, "method": "one FP64 context per instance, one block of "
                            f"{BATCH_STEPS} steps; per size class one instance timed (wall clock around the "
                            "synchronised call), times summed over the instances"},
        "speedup_vs_sequential_fp64": seq_total / ms,
        "rel_l2_vs_fp64_after_run": errs,
        "fp64_reference": "eigenvalue-free 2x2 exponential (atus_set_bragg_stable); the reference's eigen-form "
                          "loses unitarity in the pulse tails of this sweep",
        "reference_form_norm_after_run": ref_norms,
        "tune_s": t_tune,
        "schedule": sched.strip().split("\n"),
        "classes": {f"{k[0]}D-{k[1]}": len(v) for k, v in sorted(classes.items())},
    }


# ------------------------------------------------------------------ sobmin (ground state)
SOB_N, SOB_HELD_OUT, SOB_SEED = 128, 6, 2


def run_sobmin(no_cpu=False):
    """Ground states by the Sobolev descent at 128^3 on [-16,16)^3 (trap
    (1, w_y, w_z), w ~ U[0.5, 4], g ~ logU[10, 2000], N = 1, alpha = 1/2,
    fixed step 4e-4), residual 1e-10: plain sobmin from the Thomas-Fermi guess
    against the learned guess (guess.solve_learned: the decoded guess seeds
    the descent on a condensate-sized box at the full grid's spacing, whose
    converged state, embedded, seeds the full box), on the first SOB_HELD_OUT
    draws from seed 2.  The network is trained here, on the GPU with the
    project's kernels, from the committed training set (plain-sobmin ground
    states at 64^3, atus2_b200/data)."""
    from atus2_b200 import guess

    if not os.path.exists(guess.TRAIN_FILE):
        return {"unavailable": "training set atus2_b200/data/sob_train_64.npz not generated"}
    d = np.load(guess.TRAIN_FILE)
    m, sd = guess.coef_stats(d["coef"])
    t0 = time.perf_counter()
    params, hist = guess.train(guess.features(d["params"]), (d["coef"] - m) / sd, epochs=20000, lr=2e-3)
    t_train = time.perf_counter() - t0
    H = guess.draw(SOB_HELD_OUT, SOB_SEED)
    pred = guess.predict(params, guess.features(H)) * sd + m
    rows = []
    for k, (wy, wz, g) in enumerate(H):
        _, it_tf, res_tf, t_tf, mu_tf = guess.solve(SOB_N, wy, wz, g)
        _, it_nn, res_nn, t_nn, mu_nn, ns = guess.solve_learned(SOB_N, wy, wz, g, pred[k])
        rows.append(dict(w_y=float(wy), w_z=float(wz), g=float(g), iters_tf=int(it_tf), s_tf=t_tf, mu_tf=mu_tf,
                         iters_learned=[int(i) for i in it_nn], small_box=ns, s_learned=t_nn, mu_learned=mu_nn,
                         dmu=abs(mu_nn - mu_tf), res_learned=res_nn, speedup=t_tf / t_nn))
    t_tf = float(np.mean([r["s_tf"] for r in rows]))
    t_nn = float(np.mean([r["s_learned"] for r in rows]))
    out = {
        "metric": "sobmin time-to-1e-10 (128^3, FP64)",
        "value": t_tf,
        "unit": "s",
        "iterations_mean": float(np.mean([r["iters_tf"] for r in rows])),
        "learned_guess": {"value": t_nn, "unit": "s", "speedup": t_tf / t_nn,
                          "min_speedup": float(min(r["speedup"] for r in rows)),
                          "max_abs_dmu": float(max(r["dmu"] for r in rows)),
                          "method": "decoded guess -> descent on a condensate-sized box (full-grid spacing) -> "
                                    "embedded in the full box -> descent to 1e-10"},
        "training": {"draws": int(len(d["params"])), "grid": int(d["n"]), "seconds": t_train,
                     "loss_first_last": [float(hist[0]), float(hist[-1])], "epochs": len(hist)},
        "held_out": rows,
        "step": guess.STEP,
    }
    if not no_cpu:
        wy, wz, g = H[0]
        r = time_ref_sobmin(wy, wz, g)
        if r is not None:
            out["cpu_baseline"] = {"value": r["per_iter_s"] * out["iterations_mean"], "unit": "s",
                                   "cores": r["cores"], "kind": "reference",
                                   "per_iteration_s": r["per_iter_s"],
                                   "sample": f"ATUS-2 sobmin (oracle/_ref, shim FFT) at 128^3 on {r['cores']} threads, "
                                             f"held-out draw 0, {r['iters']} iterations timed from the program's own "
                                             "per-iteration output lines (set-up excluded), per-iteration time x the "
                                             "mean plain iteration count of the GPU runs"}
    return out


def time_ref_sobmin(wy, wz, g, seconds=15.0):
    """Per-iteration wall time of the reference sobmin program at 128^3 on all
    host cores: the program prints one line per iteration ("--- k"); the
    time between the first and the last line read within `seconds` (after
    the first iteration) over the iterations between them.  The run is then
    stopped (the residual target 1e-10 would take hours)."""
    prog = _ref_prog("sobmin")
    if prog is None:
        return None
    from atus2_b200 import guess

    wy, wz, g = float(wy), float(wz), float(g)  # plain floats: numpy scalars repr as np.float64(...)
    cores = os.cpu_count() or 1
    h = guess.header(SOB_N)
    V = guess.potential(h, wy, wz)
    tf = np.abs(guess.tf_guess(h, V, g))
    i = np.unravel_index(int(np.argmax(tf)), tf.shape)
    mu_tf = float(g * tf[i] ** 2 + V[i])  # the Thomas-Fermi mu: mu - V = g |psi|^2 inside the cloud
    vexpr = f"0.5*(x^2+{wy * wy!r}*y^2+{wz * wz!r}*z^2)"
    m = f"({mu_tf!r}-{vexpr})"
    half = guess.L_BOX / 2
    axes = "".join(f"<N{a}>{SOB_N}</N{a}><{a}MIN>{-half!r}</{a}MIN><{a}MAX>{half!r}</{a}MAX>" for a in "XYZ")
    xml = f"""<SIMULATION>
  <DIM>3</DIM><FILENAME>final.bin</FILENAME>
  <GUESS_3D>sqrt((abs{m}+{m})/{2 * g!r})</GUESS_3D>
  <POTENTIAL_3D>{vexpr}</POTENTIAL_3D>
  <CONSTANTS><epsilon>{guess.EPS!r}</epsilon><stepsize>{guess.STEP!r}</stepsize></CONSTANTS>
  <VCONSTANTS><Alpha_1>{guess.ALPHA!r}</Alpha_1><GS_1>{g!r}</GS_1><N>1</N></VCONSTANTS>
  <ALGORITHM>{axes}</ALGORITHM>
</SIMULATION>"""
    env = dict(os.environ, MY_NO_OF_THREADS=str(cores), OMP_NUM_THREADS=str(cores))
    stamps = []
    with tempfile.TemporaryDirectory() as tmp:
        open(os.path.join(tmp, "run.xml"), "w").write(xml)
        proc = subprocess.Popen([prog, "run.xml"], cwd=tmp, env=env, stdout=subprocess.PIPE,
                                stderr=subprocess.DEVNULL, text=True, bufsize=1)
        try:
            t_end = None
            for line in proc.stdout:
                if line.startswith("--- "):
                    now = time.perf_counter()
                    stamps.append(now)
                    if t_end is None:
                        t_end = now + seconds
                    elif now >= t_end:
                        break
        finally:
            proc.kill()
            proc.wait()
    if len(stamps) < 3:
        return None
    return {"per_iter_s": (stamps[-1] - stamps[0]) / (len(stamps) - 1), "iters": len(stamps) - 1, "cores": cores}


# ------------------------------------------------------------------ reference arm
def reference_arm(args, rank, ws, dist):
    """The reference bragg program on this host's cores: runs of W and W + K
    Strang steps (W = --warmup, K = --steps), three repeats each; the K-step
    cost is the difference of the medians, so the `steps` printed are the
    steps timed."""
    if rank != 0:
        return
    w, k = args.warmup, args.steps
    cb = run_cpu_baseline(n_short=w, n_long=w + k, repeats=3)
    if cb is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/bragg is not built (needs the ATUS-2 sources)"}))
        return
    per_step_s = N ** 3 / cb["value"]
    out = {
        "impl": "reference",
        "metric": METRIC,
        "value": cb["value"],
        "unit": UNIT,
        "n_gpus": ws,
        "steps": k,
        "warmup": w,
        "ms_per_step": per_step_s * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded Thomas-Fermi state)",
        "config": {"workload": "3D two-component Bragg pulse (bragg_ad), 256^3 on [-32,32)^3, g=100, k_L=4, delta=16, "
                               "Omega peak 8, sigma_t 0.5, dt=1e-3; reference CPU program",
                   "grid": [N, N, N], "components": 2,
                   "fft": cb["fft"],
                   "timing": f"runs of {w} and {w + k} bragg_ad steps, 3 repeats each; "
                             f"{k}-step time = difference of the medians"},
        "value_range": cb["value_range"],
        "seconds": cb["seconds"],
        "cpu_baseline": {kk: cb[kk] for kk in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def profile_block(which):
    """fp64 / mixed: one block of 2 Strang steps on the 256^3 two-component
    Bragg state, no warm-up: pass2_kernel launches in order FFT_z, FFT_y, x
    kinetic (half), IFFT_y, z potential, FFT_y, x kinetic, IFFT_y, z
    potential, FFT_y, x kinetic (half), IFFT_y, IFFT_z.  rt1d: one block of
    1000 steps of the 1D rt_solver workload (one block1d_kernel launch).
    slit / slit-mixed: one block of 2 steps of the 2048^2 double slit:
    pass3_kernel launches FFT_y, x kinetic (half), y potential, x kinetic,
    y potential, x kinetic (half), IFFT_y."""
    import torch

    from atus2_b200 import PREC_FP64, PREC_MIXED, STEP_NL, Solver

    stream = torch.cuda.Stream()
    if which == "rt1d":
        # one 1000-step block of the 1D rt_solver workload: one block1d_kernel launch
        h, psi, V = config1_inputs()
        s = Solver(h, 1, PREC_FP64)
        s.set_stream(stream.cuda_stream)
        s.set_psi(0, psi)
        s.set_alpha(0, [0.5])
        s.set_gs([10.0])
        s.set_potential(0, V)
        s.set_dt(DT)
        torch.cuda.synchronize()
        l0 = s.launches
        t0 = time.perf_counter()
        s.block(C1_NK, STEP_NL)
        s.synchronize()
        ms, launches = (time.perf_counter() - t0) * 1e3, s.launches - l0
    elif which.startswith("slit"):
        h, psi, V = config2_inputs()
        s = _c2_solver(PREC_MIXED if which == "slit-mixed" else PREC_FP64, stream, h, psi, V)
        torch.cuda.synchronize()
        l0 = s.launches
        t0 = time.perf_counter()
        s.block(2, STEP_NL)
        s.synchronize()
        ms, launches = (time.perf_counter() - t0) * 1e3, s.launches - l0
    else:
        s, ms, launches, _ = run_gpu(PREC_FP64 if which == "fp64" else PREC_MIXED, 2, 0, stream)
    s.close()
    print(json.dumps({"profile_block": which, "ms": ms, "launches": launches}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="atus", choices=["atus", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-sweep variant")
    ap.add_argument("--no-sobmin", action="store_true", help="skip the ground-state variant")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the 10^4-step accuracy runs")
    ap.add_argument("--no-configs", action="store_true", help="skip the 1D and 2D workloads")
    ap.add_argument("--file-output", action="store_true",
                    help="also time the drop-in bragg program with output every block (async vs sync files)")
    ap.add_argument("--phase-scans", action="store_true",
                    help="also time the drop-in bragg program's phase scans side by side against one by one")
    ap.add_argument("--profile-block", choices=["fp64", "mixed", "rt1d", "slit", "slit-mixed"],
                    help="run one 2-step block of the 256^3 Bragg workload (fp64, mixed; the fifth "
                         "pass2_kernel launch is the z potential pass), one 1000-step block of the 1D "
                         "rt_solver workload (rt1d) or one 2-step block of the 2048^2 double slit "
                         "(slit, slit-mixed) and exit -- for profiler captures")
    args = ap.parse_args()
    if args.profile_block:
        profile_block(args.profile_block)
        return
    args.warmup = max(args.warmup, 3)
    rank, ws, local, dist = dist_init()
    try:
        if args.impl == "reference":
            reference_arm(args, rank, ws, dist)
        else:
            atus_arm(args, rank, ws, local, dist)
    finally:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
