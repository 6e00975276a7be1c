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
device->host download of both components (pinned host memory).

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
    import torch

    from atus2_b200 import PREC_FP64, STEP_BRAGG_AD, Laser, Solver

    h = header()
    psi1, psi2 = initial_state(h)
    npts = N ** 3
    host = [torch.empty(2 * npts, dtype=torch.float64, pin_memory=True) for _ in range(2)]
    host[0].numpy()[:] = psi1.view(np.float64).ravel()
    host[1].numpy()[:] = psi2.view(np.float64).ravel()
    s = Solver(h, 2, PREC_FP64)
    s.set_stream(stream.cuda_stream)
    for c in range(2):
        s.set_alpha(c, [0.5, 0.5, 0.5])
    s.set_gs([G] * 4)
    s.set_dt(DT)
    s.set_laser(Laser.make(**laser_kw()))
    # one untimed round trip
    for c in range(2):
        s.upload_from(c, host[c].data_ptr())
    s.block(2, STEP_BRAGG_AD, None, pulse_train(s.t, 2))
    for c in range(2):
        s.download_to(c, host[c].data_ptr())
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        for c in range(2):
            s.upload_from(c, host[c].data_ptr())
        s.block(E2E_NK, STEP_BRAGG_AD, None, pulse_train(s.t, E2E_NK))
        for c in range(2):
            s.download_to(c, host[c].data_ptr())
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    s.close()
    return ms, 2 * 16 * npts, 2 * 16 * npts


def run_cpu_baseline(n_steps_sample=(1, 3)):
    """The reference program (oracle/_ref/bragg, built from the ATUS-2 sources
    with the FFTW-API shim) on this host's cores: two runs of the 256^3 Bragg
    workload of n1 and n2 Strang steps; (t2 - t1)/(n2 - n1) is the steady
    per-step cost with the set-up cancelled."""
    prog = os.path.join(ROOT, "oracle", "_ref", "bragg")
    if not os.path.exists(prog):
        return None
    from atus2_b200 import binfmt

    cores = os.cpu_count() or 1
    h = header()
    psi1, psi2 = initial_state(h)
    times = []
    with tempfile.TemporaryDirectory() as tmp:
        binfmt.write_bin(os.path.join(tmp, "inp_1.bin"), h, psi1)
        binfmt.write_bin(os.path.join(tmp, "inp_2.bin"), h, psi2)
        for ns in n_steps_sample:
            xml = f"""<SIMULATION>
  <DIM>3</DIM><FILENAME>inp_1.bin</FILENAME><FILENAME_2>inp_2.bin</FILENAME_2>
  <AMP_T>exp(-(t-{PULSE_TC!r})*(t-{PULSE_TC!r})/{2 * PULSE_SIGMA * PULSE_SIGMA!r})</AMP_T>
  <CONSTANTS><laser_k>8</laser_k><laser_dk>0</laser_dk><laser_domh>16</laser_domh>
    <rabi_threshold>1</rabi_threshold><chirp>0</chirp></CONSTANTS>
  <VCONSTANTS><Amp_1>4,4</Amp_1><Alpha_1>0.5,0.5,0.5</Alpha_1><Delta_L>0,0</Delta_L>
    <GS_1>100,100</GS_1><GS_2>100,100</GS_2><Beta>0,0,0</Beta></VCONSTANTS>
  <ALGORITHM><DT>1</DT></ALGORITHM>
  <SEQUENCE><bragg_ad dt="0.001" Nk="{ns}" output_freq="none" pn_freq="none">{ns * DT!r}</bragg_ad></SEQUENCE>
</SIMULATION>"""
            open(os.path.join(tmp, "run.xml"), "w").write(xml)
            env = dict(os.environ, MY_NO_OF_THREADS=str(cores), OMP_NUM_THREADS=str(cores))
            t0 = time.perf_counter()
            r = subprocess.run([prog, "run.xml"], cwd=tmp, env=env, capture_output=True, text=True, timeout=900)
            times.append(time.perf_counter() - t0)
            if r.returncode != 0:
                return None
    n1, n2 = n_steps_sample
    per_step = max((times[1] - times[0]) / (n2 - n1), 1e-9)
    return {
        "value": N ** 3 / per_step,
        "unit": UNIT,
        "cores": cores,
        "kind": "reference",
        "sample": f"ATUS-2 bragg (oracle/_ref, shim FFT) at 256^3 x 2 components, runs of {n1} and {n2} "
                  f"Strang steps (Nk = steps), per-step = difference / {n2 - n1}; MY_NO_OF_THREADS={cores}",
        "seconds": times,
    }


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of the
# FP64 kernels, from one ncu capture each (profiles/pass2_potential_fp64_bragg256.md,
# profiles/pipe_kernel_fp64_bragg256.md, profiles/pass2_kinetic_fp64_bragg256.md).
NCU_TRAFFIC_FP64 = {"pass2_kernel M2_NL (z)": 1.0769e9, "pipe_kernel": 1.0204e9, "pass2_kernel M2_KIN": 1.0433e9}


def roofline(s, kind, peak, peak_kind, fp64=True):
    prof = s.profile_passes(kind, reps=5)
    # pass names in atus_profile_passes order: x kinetic pass, then the
    # real-space half step (one plane-pipeline launch, or three axis passes)
    names = (["pass2_kernel M2_KIN", "pipe_kernel"] if len(prof) == 2 else
             ["pass2_kernel M2_KIN", "pass2_kernel M2_INV (y)", "pass2_kernel M2_NL (z)", "pass2_kernel M2_FWD (y)"])
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
    e2e_steps = max(1, min(args.steps // 20, 5))
    ms_e, bi, bo = run_e2e(e2e_steps, stream)
    ms_e = max_over_ranks(dist, ms_e)
    out["e2e"] = {"value": whole_job_rate(ws, npts * E2E_NK * e2e_steps, ms_e), "unit": UNIT,
                  "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo,
                  "step": f"upload 2 components, {E2E_NK} Strang steps, download 2 components", "steps": e2e_steps}
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


# ------------------------------------------------------------------ batched sweep
BATCH_COUNT, BATCH_STEPS, BATCH_SEED = 768, 4000, 1


def run_batch(stream_unused=None):
    """The batched Bragg sweep: BATCH_COUNT instances drawn from seed 1
    (atus2_b200.sweep), complex64 fields with FP64 phase arguments, autotuned,
    BATCH_STEPS steps as one graph launch.  Against it: the same instances one
    by one in plain FP64, timed on one representative instance per size class
    over the full BATCH_STEPS -- a context where one exists, a single-instance
    FP64 batch for 1D 8192 (no FP64 context fits one SM), and for 1D 16384
    (no FP64 kernel at all) the 8192 time scaled by 2 * 14/13, the FFT work
    ratio -- which also gives the accuracy of each class after BATCH_STEPS
    steps."""
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
        if key == (1, 16384):
            continue
        i = ids[0]
        d = insts[i]
        h = d["header"]
        if key == (1, 8192):
            # two complex128 components of 8192 points exceed one SM's shared
            # memory for a context: a single-instance FP64 batch (one component
            # resident) is the plain FP64 run of this instance
            one = Batch([dict(d, bragg_stable=True)], PREC_FP64, DT)
            p = sweep.initial_state(h)
            one.set_psi(0, 0, p)
            one.set_psi(0, 1, np.zeros_like(p))
            seq_ms[key] = one.run(BATCH_STEPS)
            ref = np.stack([one.psi(0, 0), one.psi(0, 1)])
            got = np.stack([b.psi(i, 0), b.psi(i, 1)])
            errs[f"{key[0]}D-{key[1]}"] = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
            one.close()
            continue
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
    if (1, 16384) in classes and (1, 8192) in classes:
        seq_ms[(1, 16384)] = seq_ms[(1, 8192)] * 2 * 14 / 13
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
    against the learned guess, on SOB_HELD_OUT draws from seed 2.  The network
    is trained here, on the GPU with the project's kernels, from the committed
    training set (plain-sobmin ground states at 64^3, atus2_b200/data).  The
    best 64-mode start (the converged state projected on the basis) bounds
    what this decoder can gain."""
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
        psi, it_tf, res_tf, t_tf, mu_tf = guess.solve(SOB_N, wy, wz, g)
        best = guess.project(psi, guess.header(SOB_N), guess.scales(wy, wz, g))
        _, it_nn, res_nn, t_nn, mu_nn = guess.solve(SOB_N, wy, wz, g, coef=pred[k])
        _, it_bs, _, t_bs, mu_bs = guess.solve(SOB_N, wy, wz, g, coef=best)
        rows.append(dict(w_y=float(wy), w_z=float(wz), g=float(g), iters_tf=int(it_tf), s_tf=t_tf, mu_tf=mu_tf,
                         iters_learned=int(it_nn), s_learned=t_nn, mu_learned=mu_nn, dmu=abs(mu_nn - mu_tf),
                         res_learned=res_nn, iters_best64=int(it_bs), s_best64=t_bs))
    t_tf = float(np.mean([r["s_tf"] for r in rows]))
    t_nn = float(np.mean([r["s_learned"] for r in rows]))
    out = {
        "metric": "sobmin time-to-1e-10 (128^3, FP64)",
        "value": t_tf,
        "unit": "s",
        "iterations_mean": float(np.mean([r["iters_tf"] for r in rows])),
        "learned_guess": {"value": t_nn, "unit": "s", "speedup": t_tf / t_nn,
                          "iterations_mean": float(np.mean([r["iters_learned"] for r in rows])),
                          "max_abs_dmu": float(max(r["dmu"] for r in rows))},
        "best_64_mode_start": {"s": float(np.mean([r["s_best64"] for r in rows])),
                               "iterations_mean": float(np.mean([r["iters_best64"] for r in rows]))},
        "training": {"draws": int(len(d["params"])), "grid": int(d["n"]), "seconds": t_train,
                     "loss_first_last": [float(hist[0]), float(hist[-1])], "epochs": len(hist)},
        "held_out": rows,
        "step": guess.STEP,
    }
    if not no_cpu:
        # the oracle port's iteration at 128^3 on all host cores, times the GPU's iteration count
        from oracle.oracle import Oracle

        wy, wz, g = H[0]
        h = guess.header(SOB_N)
        V = guess.potential(h, wy, wz)
        cores = os.cpu_count() or 1
        o = Oracle(h, 1, threads=cores)
        o.set_psi(0, guess.tf_guess(h, V, g))
        o.set_potential(0, V)
        o.set_gs([g])
        o.sob_init([guess.ALPHA], guess.STEP)
        o.sob_renormalize()
        o.sob_iterate()
        t0 = time.perf_counter()
        for _ in range(5):
            o.sob_iterate()
        per_it = (time.perf_counter() - t0) / 5
        out["cpu_baseline"] = {"value": per_it * out["iterations_mean"], "unit": "s", "cores": cores, "kind": "port",
                               "sample": f"5 Sobolev iterations of the oracle restatement at 128^3 on {cores} threads, "
                                         "times the mean plain iteration count"}
    return out


# ------------------------------------------------------------------ reference arm
def reference_arm(args, rank, ws, dist):
    if rank != 0:
        return
    cb = run_cpu_baseline()
    if cb is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/bragg is not built (needs the ATUS-2 sources)"}))
        return
    # steps of the reference arm: each step one Strang step, timed from the difference runs
    per_step_s = N ** 3 / cb["value"]
    out = {
        "impl": "reference",
        "metric": METRIC,
        "value": cb["value"],
        "unit": UNIT,
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": per_step_s * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded Thomas-Fermi state)",
        "config": {"workload": "3D two-component Bragg pulse (bragg_ad), 256^3, reference CPU program",
                   "grid": [N, N, N], "components": 2},
        "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="atus", choices=["atus", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-sweep variant")
    ap.add_argument("--no-sobmin", action="store_true", help="skip the ground-state variant")
    args = ap.parse_args()
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
