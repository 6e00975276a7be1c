"""Generates the golden fixtures in this folder from the reference programs.

Runs ATUS-2's own ``rt_solver``, ``bragg``, ``double_bragg``, ``bragg_ds``,
``raman`` and ``sobmin`` (built unmodified
from the ATUS-2 sources by ``make -C oracle ref REF=<tree>``) single-threaded on small
seeded inputs, and stores inputs and outputs as ``<case>.npz``.  The CPU tests
replay every case on the oracle restatement and require bit-identical results;
the GPU tests use the same inputs.

Usage (needs the reference programs in oracle/_ref, or the ATUS-2 source
tree named by ATUS2_REFERENCE_TREE to build them):

    python tests/golden/make_golden.py            # all cases
"""
from __future__ import annotations

import json
import math
import os
import re
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from atus2_b200 import binfmt  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(ROOT, "oracle", "_ref")


def grid(header):
    dim = int(header["nDims"])
    axes = [binfmt.x_coords(header, a) for a in range(dim)]
    return np.meshgrid(*axes, indexing="ij")


def libm(f, arr):
    """Element-wise libm call (the reference's expression parser calls libm)."""
    flat = np.asarray(arr, dtype=np.float64).ravel()
    return np.array([f(float(v)) for v in flat]).reshape(np.shape(arr))


# ------------------------------------------------------------------- cases
def rt_case(name, dim, n, lo, hi, g, alpha, V_expr, V_fn, seq, psi_fn, algo_dt):
    return dict(name=name, program="rt_solver", dim=dim, ncomp=1, n=n, lo=lo, hi=hi,
                gs=[g], Alpha_1=alpha, V_expr=V_expr, V_fn=V_fn, sequence=seq,
                psi_fn=psi_fn, algo_dt=algo_dt)


def psi_gauss_1d(X, rng):
    (x,) = X
    p = libm(math.exp, (-0.5 * (x - 1.5)) * (x - 1.5)) * np.exp(2j * x)
    return p + 1e-6 * (rng.standard_normal(x.shape) + 1j * rng.standard_normal(x.shape))


def psi_gauss_2d(X, rng):
    x, y = X
    p = libm(math.exp, -((x + 2.0) * (x + 2.0) + y * y) / 8.0) * np.exp(3j * x)
    return p + 1e-6 * (rng.standard_normal(x.shape) + 1j * rng.standard_normal(x.shape))


def psi_gauss_3d(X, rng):
    x, y, z = X
    p = libm(math.exp, -0.5 * (x * x + y * y + z * z)) * np.exp(1j * (x + 0.5 * y))
    return p + 1e-6 * (rng.standard_normal(x.shape) + 1j * rng.standard_normal(x.shape))


def psi_tf_3d(X, rng):
    x, y, z = X
    return np.sqrt(np.maximum(0.0, 2.0 - 0.5 * (x * x + y * y + z * z))).astype(np.complex128)


CASES = [
    rt_case("rt1d", 1, [128], [-16.0], [16.0], 10.0, [0.5], "0.5*x*x",
            lambda X: (0.5 * X[0]) * X[0],
            [dict(name="freeprop", dt=0.001, Nk=40, duration=0.08)], psi_gauss_1d, 1.0),
    rt_case("rt1d_tables_at_ctor", 1, [128], [-16.0], [16.0], 10.0, [0.5], "0.5*x*x",
            lambda X: (0.5 * X[0]) * X[0],
            [dict(name="freeprop", dt=0.001, Nk=40, duration=0.08)], psi_gauss_1d, 0.001),
    rt_case("rt2d_slit", 2, [64, 32], [-16.0, -8.0], [16.0, 8.0], 1.0, [0.5, 0.5],
            "200*rect(x,-0.5,0.5)*(1-rect(y,-4.5,-3.5)-rect(y,3.5,4.5))",
            None,
            [dict(name="freeprop", dt=0.0005, Nk=30, duration=0.03)], psi_gauss_2d, 1.0),
    rt_case("rt3d", 3, [16, 8, 16], [-4.0, -4.0, -4.0], [4.0, 4.0, 4.0], 5.0, [0.5, 0.5, 0.5],
            "0.5*(x*x+y*y+z*z)", lambda X: 0.5 * ((X[0] * X[0] + X[1] * X[1]) + X[2] * X[2]),
            [dict(name="freeprop", dt=0.001, Nk=20, duration=0.04)], psi_gauss_3d, 1.0),
]

BRAGG_CASES = [
    dict(name="bragg1d", dim=1, n=[256], lo=[-32.0], hi=[32.0], laser_k=2.0, laser_domh=8.0, Amp=4.0,
         tc=0.03, two_sigma2=2 * 0.01 ** 2, g=[100.0, 100.0, 100.0, 100.0], Delta_L=[0.0, 0.0], Beta=[0.0]),
    dict(name="bragg2d", dim=2, n=[64, 32], lo=[-16.0, -8.0], hi=[16.0, 8.0], laser_k=2.0, laser_domh=8.0,
         Amp=4.0, tc=0.03, two_sigma2=2 * 0.01 ** 2, g=[100.0, 100.0, 100.0, 100.0], Delta_L=[0.0, 0.5],
         Beta=[0.1, 0.0]),
    dict(name="bragg3d", dim=3, n=[16, 8, 16], lo=[-8.0, -4.0, -8.0], hi=[8.0, 4.0, 8.0], laser_k=1.5,
         laser_domh=4.0, Amp=4.0, tc=0.03, two_sigma2=2 * 0.01 ** 2, g=[100.0, 100.0, 100.0, 100.0],
         Delta_L=[0.0, 0.0], Beta=[0.0, 0.0, 0.0]),
]

DBRAGG_CASES = [
    dict(name="dbragg1d", dim=1, n=[256], lo=[-32.0], hi=[32.0], laser_k=2.0, laser_domh=8.0, Amp=4.0,
         tc=0.03, two_sigma2=2 * 0.01 ** 2, g=[100.0, 90.0, 90.0, 90.0, 100.0, 95.0, 90.0, 95.0, 100.0],
         Delta_L=[0.0, 0.0, 0.0], Beta=[0.05]),
    dict(name="dbragg2d", dim=2, n=[64, 32], lo=[-16.0, -8.0], hi=[16.0, 8.0], laser_k=2.0, laser_domh=8.0,
         Amp=4.0, tc=0.03, two_sigma2=2 * 0.01 ** 2, g=[100.0] * 9, Delta_L=[0.0, 0.5, 0.5], Beta=[0.1, 0.05]),
    dict(name="dbragg3d", dim=3, n=[16, 8, 16], lo=[-8.0, -4.0, -8.0], hi=[8.0, 4.0, 8.0], laser_k=1.5,
         laser_domh=4.0, Amp=4.0, tc=0.03, two_sigma2=2 * 0.01 ** 2, g=[100.0] * 9, Delta_L=[0.0, 0.0, 0.0],
         Beta=[0.0, 0.02, 0.03]),
]

# two species (bragg_ds): g is the 4 x 4 matrix row by row (GS_1..GS_4)
_G4 = [100.0, 90.0, 20.0, 15.0, 90.0, 95.0, 15.0, 20.0, 20.0, 15.0, 80.0, 70.0, 15.0, 20.0, 70.0, 75.0]
BRAGGDS_CASES = [
    dict(name="braggds1d", dim=1, n=[256], lo=[-32.0], hi=[32.0], laser_k=2.0, laser_k_2=1.5, laser_domh=8.0,
         laser_domh_2=4.5, laser_dk=0.2, laser_dk_2=0.3, Amp=4.0, Amp_2=3.0, durations=[0.0305, 0.0505], g=_G4,
         Delta_L=[0.0, 0.3, 0.0, -0.2], Beta=[0.05], Beta_2=[-0.03], Alpha_2=0.35),
    dict(name="braggds2d", dim=2, n=[64, 32], lo=[-16.0, -8.0], hi=[16.0, 8.0], laser_k=2.0, laser_k_2=1.5,
         laser_domh=8.0, laser_domh_2=4.5, laser_dk=0.2, laser_dk_2=0.3, Amp=4.0, Amp_2=3.0,
         durations=[0.0505, 0.0305], g=_G4, Delta_L=[0.0, 0.5, 0.1, 0.4], Beta=[0.1, 0.0], Beta_2=[0.02, 0.0],
         Alpha_2=0.35),
    dict(name="braggds3d", dim=3, n=[16, 8, 16], lo=[-8.0, -4.0, -8.0], hi=[8.0, 4.0, 8.0], laser_k=1.5,
         laser_k_2=1.0, laser_domh=4.0, laser_domh_2=2.0, laser_dk=0.0, laser_dk_2=0.1, Amp=4.0, Amp_2=3.0,
         durations=[0.0305, 0.0505], g=_G4, Delta_L=[0.0, 0.0, 0.0, 0.0], Beta=[0.0, 0.0, 0.0],
         Beta_2=[0.01, 0.0, 0.0], Alpha_2=0.35),
]

# the numerical steps of CRT_Base_IF ("raman", "bragg"): GSL eigensolver in
# the reference, the shim's Jacobi solver in the oracle build
_G3 = [100.0, 90.0, 80.0, 90.0, 95.0, 85.0, 80.0, 85.0, 90.0]
_NUM_SEQ = [dict(name="raman", dt=0.001, Nk=10, duration=0.04, rabi=True),
            dict(name="bragg", dt=0.001, Nk=10, duration=0.03, rabi=True),
            dict(name="freeprop", dt=0.001, Nk=10, duration=0.02, rabi=True)]
NUM_CASES = [
    dict(name="raman1d", program="raman", dim=1, n=[256], lo=[-32.0], hi=[32.0], laser_k=2.0, laser_domh=10.0,
         laser_dk=0.0, Amp=[8.0, 6.0], chirp=0.0, g=_G3, Delta_L=[0.0, 0.5, -0.5], Beta=[0.05], seq=_NUM_SEQ),
    dict(name="raman2d", program="raman", dim=2, n=[64, 32], lo=[-16.0, -8.0], hi=[16.0, 8.0], laser_k=2.0,
         laser_domh=10.0, laser_dk=0.0, Amp=[8.0, 6.0], chirp=0.0, g=_G3, Delta_L=[0.0, 0.5, -0.5],
         Beta=[0.1, 0.05], seq=_NUM_SEQ),
    dict(name="raman3d", program="raman", dim=3, n=[16, 8, 16], lo=[-8.0, -4.0, -8.0], hi=[8.0, 4.0, 8.0],
         laser_k=1.5, laser_domh=10.0, laser_dk=0.0, Amp=[8.0, 6.0], chirp=0.0, g=_G3, Delta_L=[0.0, 0.5, -0.5],
         Beta=[0.02, 0.03, -0.01], seq=_NUM_SEQ),
    dict(name="nbragg2d", program="bragg", dim=2, n=[64, 32], lo=[-16.0, -8.0], hi=[16.0, 8.0], laser_k=2.0,
         laser_domh=8.0, laser_dk=0.0, Amp=[4.0, 3.0], chirp=0.0, g=[100.0, 90.0, 90.0, 95.0],
         Delta_L=[0.0, 0.3], Beta=[0.1, 0.05],
         seq=[dict(name="bragg", dt=0.001, Nk=10, duration=0.05, rabi=True),
              dict(name="freeprop", dt=0.001, Nk=10, duration=0.02, rabi=True)]),
]

# phase scans (CRT_Base_IF::run_sequence, chirp_mode 1): no_of_chirps runs of
# the same sequence from the same start, scan s with laser phase s 2 pi / n
# and the chirp rates chirp_min, chirp_max, then midpoints (include/
# CRT_Base_IF.h:755-921)
PHASESCAN_CASES = [
    dict(name="scan1d", dim=1, n=[256], lo=[-32.0], hi=[32.0], laser_k=2.0, laser_domh=8.0, Amp=4.0,
         tc=0.02, two_sigma2=2 * 0.008 ** 2, g=[100.0, 90.0, 90.0, 100.0], Delta_L=[0.0, 0.2], Beta=[0.05],
         chirps=5, chirp_min=-2.0, chirp_max=3.0),
    dict(name="scan2d", dim=2, n=[64, 32], lo=[-16.0, -8.0], hi=[16.0, 8.0], laser_k=2.0, laser_domh=8.0,
         Amp=4.0, tc=0.02, two_sigma2=2 * 0.008 ** 2, g=[100.0] * 4, Delta_L=[0.0, 0.5], Beta=[0.1, 0.0],
         chirps=4, chirp_min=-1.0, chirp_max=1.0),
]

SOB_CASES = [
    dict(name="sob1d", dim=1, n=[64], lo=[-8.0], hi=[8.0], g=50.0, Nparticles=1.0, alpha=0.5, stepsize=0.01,
         epsilon=1e-7, V_expr="0.5*x*x", guess_expr="exp(-0.5*x*x)"),
    dict(name="sob2d", dim=2, n=[32, 32], lo=[-6.0, -6.0], hi=[6.0, 6.0], g=20.0, Nparticles=1.0, alpha=0.5,
         stepsize=0.01, epsilon=1e-6, V_expr="0.5*(x*x+4*y*y)", guess_expr="exp(-0.5*(x*x+y*y))"),
    dict(name="sob3d", dim=3, n=[16, 16, 8], lo=[-6.0, -6.0, -6.0], hi=[6.0, 6.0, 6.0], g=10.0,
         Nparticles=1.0, alpha=0.5, stepsize=0.01, epsilon=1e-5, V_expr="0.5*(x*x+y*y+z*z)",
         guess_expr="exp(-0.5*(x*x+y*y+z*z))"),
]


# --------------------------------------------------------------- helpers
def xml_vec(v):
    return ",".join(repr(float(a)) for a in v)


def run(prog, cwd):
    env = dict(os.environ, MY_NO_OF_THREADS="1", OMP_NUM_THREADS="1")
    r = subprocess.run([os.path.join(REF, prog), "run.xml"], cwd=cwd, capture_output=True, text=True,
                       env=env, timeout=600)
    if r.returncode != 0:
        raise RuntimeError(f"{prog} failed: {r.stdout[-2000:]} {r.stderr[-2000:]}")
    return r.stdout


def seq_xml(seq, extra=""):
    def dur(d):
        return ",".join(repr(float(v)) for v in d) if isinstance(d, (list, tuple)) else repr(d)

    return "".join(
        f'<{s["name"]} dt="{s["dt"]!r}" Nk="{s["Nk"]}" output_freq="each" pn_freq="each"{extra if s.get("rabi") else ""}>'
        f'{dur(s["duration"])}</{s["name"]}>' for s in seq)


def collect_outputs(cwd, ncomp, seq):
    """Every block's Save_Phi output, in order of time."""
    files = {}
    for fn in os.listdir(cwd):
        m = re.match(r"^(-?\d+\.\d{3})_(\d)\.bin$", fn)
        if m and fn != "inp_1.bin":
            files.setdefault(m.group(1), {})[int(m.group(2))] = fn
    out_t, out_psi = [], []
    for key in sorted(files, key=float):
        comps = files[key]
        recs = [binfmt.read_bin(os.path.join(cwd, comps[c + 1])) for c in range(ncomp)]
        out_t.append(float(recs[0].header["t"]))
        out_psi.append(np.stack([r.data for r in recs]))
    return np.array(out_t), np.stack(out_psi)


def make_rt(case, tmp):
    rng = np.random.default_rng(0)
    h = binfmt.make_header(case["dim"], case["n"], case["lo"], case["hi"], dt=0.001)
    X = grid(h)
    psi0 = case["psi_fn"](X, rng)
    binfmt.write_bin(os.path.join(tmp, "inp_1.bin"), h, psi0)
    xml = f"""<SIMULATION>
  <DIM>{case['dim']}</DIM>
  <FILENAME>inp_1.bin</FILENAME>
  <POTENTIAL_{case['dim']}D>{case['V_expr']}</POTENTIAL_{case['dim']}D>
  <CONSTANTS><unused>0</unused></CONSTANTS>
  <VCONSTANTS><Alpha_1>{xml_vec(case['Alpha_1'])}</Alpha_1><GS_1>{xml_vec(case['gs'])}</GS_1></VCONSTANTS>
  <ALGORITHM><DT>{case['algo_dt']!r}</DT></ALGORITHM>
  <SEQUENCE>{seq_xml(case['sequence'])}</SEQUENCE>
</SIMULATION>"""
    open(os.path.join(tmp, "run.xml"), "w").write(xml)
    run("rt_solver", tmp)
    t, psi = collect_outputs(tmp, 1, case["sequence"])
    if case["dim"] == 2 and case["V_fn"] is None:
        V = potential_2d_from_txt(os.path.join(tmp, "potential.txt"), h)
    else:
        V = case["V_fn"](X)
    params = dict(program="rt_solver", dim=case["dim"], ncomp=1, header_dt=0.001, algo_dt=case["algo_dt"],
                  Alpha_1=case["Alpha_1"], gs=case["gs"], sequence=case["sequence"])
    return dict(header=h.tobytes(), psi0=psi0[None], V=V, t=t, psi=psi, params=json.dumps(params), xml=xml)


def potential_2d_from_txt(path, h):
    """rt_solver writes the 2D potential to potential.txt (rt_solver.cpp:117-130)
    with 6 significant digits; the slit potential only takes the values 0 and
    200, which that format holds exactly."""
    vals = []
    for line in open(path):
        parts = line.split()
        if len(parts) == 3:
            vals.append(float(parts[2]))
    nx, ny = int(h["nDimX"]), int(h["nDimY"])
    V = np.array(vals).reshape(nx, ny)
    assert set(np.unique(V)).issubset({0.0, 200.0})
    return V


def make_bragg(case, tmp):
    rng = np.random.default_rng(1)
    dim = case["dim"]
    h = binfmt.make_header(dim, case["n"], case["lo"], case["hi"], dt=0.001)
    X = grid(h)
    r2 = sum(x * x for x in X)
    psi1 = np.sqrt(np.maximum(0.0, 1.0 - 0.1 * r2)) * (1 + 0.01 * rng.standard_normal(r2.shape))
    psi1 = psi1.astype(np.complex128)
    psi2 = np.zeros_like(psi1)
    binfmt.write_bin(os.path.join(tmp, "inp_1.bin"), h, psi1)
    binfmt.write_bin(os.path.join(tmp, "inp_2.bin"), h, psi2)
    seq = [dict(name="bragg_ad", dt=0.001, Nk=20, duration=0.06, rabi=True),
           dict(name="freeprop", dt=0.001, Nk=20, duration=0.04, rabi=True)]
    xml = f"""<SIMULATION>
  <DIM>{dim}</DIM>
  <FILENAME>inp_1.bin</FILENAME>
  <FILENAME_2>inp_2.bin</FILENAME_2>
  <AMP_T>exp(-(t-{case['tc']!r})*(t-{case['tc']!r})/{case['two_sigma2']!r})</AMP_T>
  <CONSTANTS>
    <laser_k>{case['laser_k']!r}</laser_k><laser_dk>0</laser_dk><laser_domh>{case['laser_domh']!r}</laser_domh>
    <rabi_threshold>1.0</rabi_threshold><chirp>0</chirp>
  </CONSTANTS>
  <VCONSTANTS>
    <Amp_1>{case['Amp']!r},{case['Amp']!r}</Amp_1>
    <Alpha_1>{xml_vec([0.5] * dim)}</Alpha_1>
    <Delta_L>{xml_vec(case['Delta_L'])}</Delta_L>
    <GS_1>{xml_vec(case['g'][:2])}</GS_1>
    <GS_2>{xml_vec(case['g'][2:])}</GS_2>
    <Beta>{xml_vec(case['Beta'])}</Beta>
  </VCONSTANTS>
  <ALGORITHM><DT>1</DT></ALGORITHM>
  <SEQUENCE>{seq_xml(seq, ' rabi_output_freq="each"')}</SEQUENCE>
</SIMULATION>"""
    open(os.path.join(tmp, "run.xml"), "w").write(xml)
    run("bragg", tmp)
    t, psi = collect_outputs(tmp, 2, seq)
    rabi = []
    for s in (1, 2):
        rows = [ln.split() for ln in open(os.path.join(tmp, f"Rabi_{s}_0.txt")) if not ln.startswith("#")]
        rabi += [[float(v) for v in r[1:]] for r in rows if r]
    k0 = np.zeros((3, dim))
    k0[1, 0] = 2 * case["laser_k"]
    k0[2, 0] = -2 * case["laser_k"]
    params = dict(program="bragg", dim=dim, ncomp=2, header_dt=0.001, algo_dt=1.0, Alpha_1=[0.5] * dim,
                  gs=case["g"], sequence=seq, AMP_T=dict(tc=case["tc"], two_sigma2=case["two_sigma2"]),
                  laser_k=case["laser_k"], laser_domh=case["laser_domh"], laser_dk=0.0, chirp=0.0,
                  Amp_1=[case["Amp"], case["Amp"]], Delta_L=case["Delta_L"], Beta=case["Beta"],
                  rabi_threshold=1.0, rabi_k0=k0.tolist())
    return dict(header=h.tobytes(), psi0=np.stack([psi1, psi2]), t=t, psi=psi, rabi=np.array(rabi),
                params=json.dumps(params), xml=xml)


def make_dbragg(case, tmp):
    """The three-level program (double_bragg): state 1 a Thomas-Fermi-like
    profile with noise, states 2 and 3 empty."""
    rng = np.random.default_rng(2)
    dim = case["dim"]
    h = binfmt.make_header(dim, case["n"], case["lo"], case["hi"], dt=0.001)
    X = grid(h)
    r2 = sum(x * x for x in X)
    psi1 = np.sqrt(np.maximum(0.0, 1.0 - 0.1 * r2)) * (1 + 0.01 * rng.standard_normal(r2.shape))
    psi1 = psi1.astype(np.complex128)
    psi2 = np.zeros_like(psi1)
    for k, p in enumerate((psi1, psi2, psi2)):
        binfmt.write_bin(os.path.join(tmp, f"inp_{k + 1}.bin"), h, p)
    seq = [dict(name="bragg_ad", dt=0.001, Nk=20, duration=0.06, rabi=True),
           dict(name="freeprop", dt=0.001, Nk=20, duration=0.04, rabi=True)]
    g = case["g"]
    xml = f"""<SIMULATION>
  <DIM>{dim}</DIM>
  <FILENAME>inp_1.bin</FILENAME>
  <FILENAME_2>inp_2.bin</FILENAME_2>
  <FILENAME_3>inp_3.bin</FILENAME_3>
  <AMP_T>exp(-(t-{case['tc']!r})*(t-{case['tc']!r})/{case['two_sigma2']!r})</AMP_T>
  <CONSTANTS>
    <laser_k>{case['laser_k']!r}</laser_k><laser_dk>0</laser_dk><laser_domh>{case['laser_domh']!r}</laser_domh>
    <rabi_threshold>1.0</rabi_threshold><chirp>0</chirp>
  </CONSTANTS>
  <VCONSTANTS>
    <Amp_1>{case['Amp']!r},{case['Amp']!r}</Amp_1>
    <Alpha_1>{xml_vec([0.5] * dim)}</Alpha_1>
    <Delta_L>{xml_vec(case['Delta_L'])}</Delta_L>
    <GS_1>{xml_vec(g[0:3])}</GS_1>
    <GS_2>{xml_vec(g[3:6])}</GS_2>
    <GS_3>{xml_vec(g[6:9])}</GS_3>
    <Beta>{xml_vec(case['Beta'])}</Beta>
  </VCONSTANTS>
  <ALGORITHM><DT>1</DT></ALGORITHM>
  <SEQUENCE>{seq_xml(seq, ' rabi_output_freq="each"')}</SEQUENCE>
</SIMULATION>"""
    open(os.path.join(tmp, "run.xml"), "w").write(xml)
    run("double_bragg", tmp)
    t, psi = collect_outputs(tmp, 3, seq)
    rabi = []
    for s in (1, 2):
        rows = [ln.split() for ln in open(os.path.join(tmp, f"Rabi_{s}_0.txt")) if not ln.startswith("#")]
        rabi += [[float(v) for v in r[1:]] for r in rows if r]
    k0 = np.zeros((3, dim))
    k0[1, 0] = 2 * case["laser_k"]
    k0[2, 0] = -2 * case["laser_k"]
    params = dict(program="double_bragg", dim=dim, ncomp=3, header_dt=0.001, algo_dt=1.0, Alpha_1=[0.5] * dim,
                  gs=g, sequence=seq, AMP_T=dict(tc=case["tc"], two_sigma2=case["two_sigma2"]),
                  laser_k=case["laser_k"], laser_domh=case["laser_domh"], laser_dk=0.0, chirp=0.0,
                  Amp_1=[case["Amp"], case["Amp"]], Delta_L=case["Delta_L"], Beta=case["Beta"],
                  rabi_threshold=1.0, rabi_k0=k0.tolist())
    return dict(header=h.tobytes(), psi0=np.stack([psi1, psi2, psi2]), t=t, psi=psi, rabi=np.array(rabi),
                params=json.dumps(params), xml=xml)


def make_bragg_ds(case, tmp):
    """The two-species program (bragg_ds): species 1 in components 1-2,
    species 2 in 3-4, a Thomas-Fermi-like profile with noise in the first
    state of each species; bragg_ad with one pulse window per species, then
    freeprop."""
    rng = np.random.default_rng(3)
    dim = case["dim"]
    h = binfmt.make_header(dim, case["n"], case["lo"], case["hi"], dt=0.001)
    X = grid(h)
    r2 = sum(x * x for x in X)
    psi1 = np.sqrt(np.maximum(0.0, 1.0 - 0.1 * r2)) * (1 + 0.01 * rng.standard_normal(r2.shape))
    psi3 = np.sqrt(np.maximum(0.0, 0.8 - 0.12 * r2)) * (1 + 0.01 * rng.standard_normal(r2.shape))
    psi1, psi3 = psi1.astype(np.complex128), psi3.astype(np.complex128)
    zero = np.zeros_like(psi1)
    psi0 = np.stack([psi1, zero, psi3, zero])
    for k in range(4):
        binfmt.write_bin(os.path.join(tmp, f"inp_{k + 1}.bin"), h, psi0[k])
    seq = [dict(name="bragg_ad", dt=0.001, Nk=10, duration=list(case["durations"]), rabi=True),
           dict(name="freeprop", dt=0.001, Nk=20, duration=0.04, rabi=True)]
    g = case["g"]
    gs_xml = "".join(f"<GS_{i + 1}>{xml_vec(g[4 * i:4 * i + 4])}</GS_{i + 1}>" for i in range(4))
    xml = f"""<SIMULATION>
  <DIM>{dim}</DIM>
  <FILENAME>inp_1.bin</FILENAME>
  <FILENAME_2>inp_2.bin</FILENAME_2>
  <FILENAME_3>inp_3.bin</FILENAME_3>
  <FILENAME_4>inp_4.bin</FILENAME_4>
  <CONSTANTS>
    <laser_k>{case['laser_k']!r}</laser_k><laser_k_2>{case['laser_k_2']!r}</laser_k_2>
    <laser_dk>{case['laser_dk']!r}</laser_dk><laser_dk_2>{case['laser_dk_2']!r}</laser_dk_2>
    <laser_domh>{case['laser_domh']!r}</laser_domh><laser_domh_2>{case['laser_domh_2']!r}</laser_domh_2>
    <rabi_threshold>1.0</rabi_threshold>
  </CONSTANTS>
  <VCONSTANTS>
    <Amp_1>{case['Amp']!r},{case['Amp']!r}</Amp_1>
    <Amp_2>{case['Amp_2']!r},{case['Amp_2']!r}</Amp_2>
    <Alpha_1>{xml_vec([0.5] * dim)}</Alpha_1>
    <Alpha_2>{xml_vec([case['Alpha_2']] * dim)}</Alpha_2>
    <Delta_L>{xml_vec(case['Delta_L'])}</Delta_L>
    {gs_xml}
    <Beta>{xml_vec(case['Beta'])}</Beta>
    <Beta_2>{xml_vec(case['Beta_2'])}</Beta_2>
  </VCONSTANTS>
  <ALGORITHM><DT>1</DT></ALGORITHM>
  <SEQUENCE>{seq_xml(seq, ' rabi_output_freq="each"')}</SEQUENCE>
</SIMULATION>"""
    open(os.path.join(tmp, "run.xml"), "w").write(xml)
    run("bragg_ds", tmp)
    t, psi = collect_outputs(tmp, 4, seq)
    rabi = []
    for s in (1, 2):
        rows = []
        for sp in (1, 2):
            fn = os.path.join(tmp, f"Spezie_{sp}_Rabi_{s}_0.txt")
            rows.append([[float(v) for v in ln.split()[1:]] for ln in open(fn) if not ln.startswith("#") and ln.split()])
        rabi += [r1 + r2 for r1, r2 in zip(*rows)]
    k0 = np.zeros((3, dim))
    k0[1, 0] = 2 * case["laser_k"]
    k0[2, 0] = -2 * case["laser_k"]
    k02 = np.zeros((3, dim))
    k02[1, 0] = 2 * case["laser_k_2"]
    k02[2, 0] = -2 * case["laser_k_2"]
    params = dict(program="bragg_ds", dim=dim, ncomp=4, header_dt=0.001, algo_dt=1.0, Alpha_1=[0.5] * dim,
                  Alpha_2=[case["Alpha_2"]] * dim, gs=g, sequence=seq,
                  laser_k=case["laser_k"], laser_domh=case["laser_domh"], laser_dk=case["laser_dk"], chirp=0.0,
                  laser_k_2=case["laser_k_2"], laser_domh_2=case["laser_domh_2"], laser_dk_2=case["laser_dk_2"],
                  Amp_1=[case["Amp"], case["Amp"]], Amp_2=[case["Amp_2"], case["Amp_2"]],
                  Delta_L=case["Delta_L"], Beta=case["Beta"], Beta_2=case["Beta_2"],
                  rabi_threshold=1.0, rabi_k0=k0.tolist(), rabi_k0_2=k02.tolist())
    return dict(header=h.tobytes(), psi0=psi0, t=t, psi=psi, rabi=np.array(rabi), params=json.dumps(params),
                xml=xml)


def make_numerical(case, tmp):
    """The numerical steps of CRT_Base_IF ("raman" three-state, "bragg"
    n-state) in the raman program (three states) or the bragg program (two):
    the first state a Thomas-Fermi-like profile with noise, the others empty."""
    rng = np.random.default_rng(4)
    dim, prog = case["dim"], case["program"]
    ncomp = 3 if prog == "raman" else 2
    h = binfmt.make_header(dim, case["n"], case["lo"], case["hi"], dt=0.001)
    X = grid(h)
    r2 = sum(x * x for x in X)
    psi1 = np.sqrt(np.maximum(0.0, 1.0 - 0.1 * r2)) * (1 + 0.01 * rng.standard_normal(r2.shape))
    psi0 = np.zeros((ncomp,) + psi1.shape, dtype=np.complex128)
    psi0[0] = psi1
    for k in range(ncomp):
        binfmt.write_bin(os.path.join(tmp, f"inp_{k + 1}.bin"), h, psi0[k])
    seq = case["seq"]
    g = case["g"]
    files = "".join(f"<FILENAME_{k + 1}>inp_{k + 1}.bin</FILENAME_{k + 1}>" for k in range(1, ncomp))
    gs_xml = "".join(f"<GS_{i + 1}>{xml_vec(g[ncomp * i:ncomp * i + ncomp])}</GS_{i + 1}>" for i in range(ncomp))
    xml = f"""<SIMULATION>
  <DIM>{dim}</DIM>
  <FILENAME>inp_1.bin</FILENAME>
  {files}
  <CONSTANTS>
    <laser_k>{case['laser_k']!r}</laser_k><laser_dk>{case['laser_dk']!r}</laser_dk>
    <laser_domh>{case['laser_domh']!r}</laser_domh>
    <rabi_threshold>1.0</rabi_threshold><chirp>{case['chirp']!r}</chirp>
  </CONSTANTS>
  <VCONSTANTS>
    <Amp_1>{xml_vec(case['Amp'])}</Amp_1>
    <Alpha_1>{xml_vec([0.5] * dim)}</Alpha_1>
    <Delta_L>{xml_vec(case['Delta_L'])}</Delta_L>
    {gs_xml}
    <Beta>{xml_vec(case['Beta'])}</Beta>
  </VCONSTANTS>
  <ALGORITHM><DT>1</DT></ALGORITHM>
  <SEQUENCE>{seq_xml(seq, ' rabi_output_freq="each"')}</SEQUENCE>
</SIMULATION>"""
    open(os.path.join(tmp, "run.xml"), "w").write(xml)
    run(prog, tmp)
    t, psi = collect_outputs(tmp, ncomp, seq)
    rabi = []
    for s in range(1, len(seq) + 1):
        rows = [ln.split() for ln in open(os.path.join(tmp, f"Rabi_{s}_0.txt")) if not ln.startswith("#")]
        rabi += [[float(v) for v in r[1:]] for r in rows if r]
    k0 = np.zeros((3, dim))
    k0[1, 0] = 2 * case["laser_k"]
    k0[2, 0] = -2 * case["laser_k"]
    params = dict(program=prog, dim=dim, ncomp=ncomp, header_dt=0.001, algo_dt=1.0, Alpha_1=[0.5] * dim,
                  gs=g, sequence=seq, laser_k=case["laser_k"], laser_domh=case["laser_domh"],
                  laser_dk=case["laser_dk"], chirp=case["chirp"], Amp_1=list(case["Amp"]),
                  Delta_L=case["Delta_L"], Beta=case["Beta"], rabi_threshold=1.0, rabi_k0=k0.tolist())
    return dict(header=h.tobytes(), psi0=psi0, t=t, psi=psi, rabi=np.array(rabi), params=json.dumps(params),
                xml=xml)


def make_phasescan(case, tmp):
    """The bragg program with a phase scan on its bragg_ad sequence
    (no_of_chirps, chirp_mode 1), Rabi sums every block, then freeprop:
    every .bin output, the Rabi file of each scan and the Chirp file."""
    rng = np.random.default_rng(5)
    dim = case["dim"]
    h = binfmt.make_header(dim, case["n"], case["lo"], case["hi"], dt=0.001)
    X = grid(h)
    r2 = sum(x * x for x in X)
    psi1 = (np.sqrt(np.maximum(0.0, 1.0 - 0.1 * r2)) * (1 + 0.01 * rng.standard_normal(r2.shape))).astype(np.complex128)
    psi2 = np.zeros_like(psi1)
    binfmt.write_bin(os.path.join(tmp, "inp_1.bin"), h, psi1)
    binfmt.write_bin(os.path.join(tmp, "inp_2.bin"), h, psi2)
    nc = case["chirps"]
    xml = f"""<SIMULATION>
  <DIM>{dim}</DIM>
  <FILENAME>inp_1.bin</FILENAME>
  <FILENAME_2>inp_2.bin</FILENAME_2>
  <AMP_T>exp(-(t-{case['tc']!r})*(t-{case['tc']!r})/{case['two_sigma2']!r})</AMP_T>
  <CONSTANTS>
    <laser_k>{case['laser_k']!r}</laser_k><laser_dk>0</laser_dk><laser_domh>{case['laser_domh']!r}</laser_domh>
    <rabi_threshold>1.0</rabi_threshold><chirp>0</chirp>
  </CONSTANTS>
  <VCONSTANTS>
    <Amp_1>{case['Amp']!r},{case['Amp']!r}</Amp_1>
    <Alpha_1>{xml_vec([0.5] * dim)}</Alpha_1>
    <Delta_L>{xml_vec(case['Delta_L'])}</Delta_L>
    <GS_1>{xml_vec(case['g'][:2])}</GS_1><GS_2>{xml_vec(case['g'][2:])}</GS_2>
    <Beta>{xml_vec(case['Beta'])}</Beta>
  </VCONSTANTS>
  <ALGORITHM><DT>1</DT></ALGORITHM>
  <SEQUENCE>
    <bragg_ad dt="0.001" Nk="10" output_freq="each" pn_freq="none" rabi_output_freq="each" no_of_chirps="{nc}"
      chirp_mode="1" chirp_min="{case['chirp_min']!r}" chirp_max="{case['chirp_max']!r}">0.04</bragg_ad>
    <freeprop dt="0.001" Nk="10" output_freq="each" pn_freq="none" rabi_output_freq="each">0.02</freeprop>
  </SEQUENCE>
</SIMULATION>"""
    open(os.path.join(tmp, "run.xml"), "w").write(xml)
    run("bragg", tmp)
    t, psi = collect_outputs(tmp, 2, [])

    def rows(path):
        return np.array([[float(v) for v in ln.split()] for ln in open(path) if not ln.startswith("#") and ln.split()])

    rabi = np.stack([rows(os.path.join(tmp, f"Rabi_1_{k}.txt")) for k in range(nc)])
    rabi_free = rows(os.path.join(tmp, "Rabi_2_0.txt"))
    chirp = rows(os.path.join(tmp, "Chirp_1.txt"))
    params = dict(program="bragg", dim=dim, ncomp=2, chirps=nc, laser_k=case["laser_k"])
    return dict(header=h.tobytes(), psi0=np.stack([psi1, psi2]), t=t, psi=psi, rabi_scans=rabi,
                rabi_free=rabi_free, chirp=chirp, params=json.dumps(params), xml=xml)


def make_sob(case, tmp):
    dim = case["dim"]
    ax = "XYZ"[:dim]
    algo = "".join(f"<N{a}>{n}</N{a}>" for a, n in zip(ax, case["n"]))
    algo += "".join(f"<{a}MIN>{lo!r}</{a}MIN><{a}MAX>{hi!r}</{a}MAX>" for a, lo, hi in zip(ax, case["lo"], case["hi"]))
    xml = f"""<SIMULATION>
  <DIM>{dim}</DIM>
  <FILENAME>final.bin</FILENAME>
  <GUESS_{dim}D>{case['guess_expr']}</GUESS_{dim}D>
  <POTENTIAL_{dim}D>{case['V_expr']}</POTENTIAL_{dim}D>
  <CONSTANTS><epsilon>{case['epsilon']!r}</epsilon><stepsize>{case['stepsize']!r}</stepsize></CONSTANTS>
  <VCONSTANTS><Alpha_1>{case['alpha']!r}</Alpha_1><GS_1>{case['g']!r}</GS_1><N>{case['Nparticles']!r}</N></VCONSTANTS>
  <ALGORITHM>{algo}</ALGORITHM>
</SIMULATION>"""
    open(os.path.join(tmp, "run.xml"), "w").write(xml)
    out = run("sobmin", tmp)
    res = [float(m) for m in re.findall(r"^res (\S+)$", out, re.M)]
    final = binfmt.read_bin(os.path.join(tmp, "final.bin"))
    params = dict(program="sobmin", dim=dim, n=case["n"], lo=case["lo"], hi=case["hi"], g=case["g"],
                  Nparticles=case["Nparticles"], alpha=case["alpha"], stepsize=case["stepsize"],
                  epsilon=case["epsilon"], V_expr=case["V_expr"], guess_expr=case["guess_expr"])
    return dict(header=final.header.tobytes(), psi=final.data, res=np.array(res), iterations=len(res),
                params=json.dumps(params), xml=xml)


def main():
    if not os.path.exists(os.path.join(REF, "raman")):
        tree = os.environ.get("ATUS2_REFERENCE_TREE")
        if not tree:
            sys.exit("oracle/_ref is not built: set ATUS2_REFERENCE_TREE to the ATUS-2 source tree")
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={tree}"], check=True)
    only = set(sys.argv[1:])
    keep = (lambda c: not only or c["name"] in only)
    global CASES, BRAGG_CASES, DBRAGG_CASES, BRAGGDS_CASES, SOB_CASES
    CASES, BRAGG_CASES = [c for c in CASES if keep(c)], [c for c in BRAGG_CASES if keep(c)]
    DBRAGG_CASES, SOB_CASES = [c for c in DBRAGG_CASES if keep(c)], [c for c in SOB_CASES if keep(c)]
    BRAGGDS_CASES = [c for c in BRAGGDS_CASES if keep(c)]
    global NUM_CASES, PHASESCAN_CASES
    NUM_CASES = [c for c in NUM_CASES if keep(c)]
    PHASESCAN_CASES = [c for c in PHASESCAN_CASES if keep(c)]
    for case in PHASESCAN_CASES:
        with tempfile.TemporaryDirectory() as tmp:
            d = make_phasescan(case, tmp)
            np.savez_compressed(os.path.join(HERE, case["name"] + ".npz"), **d)
            print("wrote", case["name"])
    for case in CASES:
        with tempfile.TemporaryDirectory() as tmp:
            d = make_rt(case, tmp)
        np.savez_compressed(os.path.join(HERE, case["name"] + ".npz"), **d)
        print("wrote", case["name"], d["psi"].shape)
    for case in BRAGG_CASES:
        with tempfile.TemporaryDirectory() as tmp:
            d = make_bragg(case, tmp)
        np.savez_compressed(os.path.join(HERE, case["name"] + ".npz"), **d)
        print("wrote", case["name"], d["psi"].shape, d["rabi"].shape)
    for case in DBRAGG_CASES:
        with tempfile.TemporaryDirectory() as tmp:
            d = make_dbragg(case, tmp)
        np.savez_compressed(os.path.join(HERE, case["name"] + ".npz"), **d)
        print("wrote", case["name"], d["psi"].shape, d["rabi"].shape)
    for case in BRAGGDS_CASES:
        with tempfile.TemporaryDirectory() as tmp:
            d = make_bragg_ds(case, tmp)
        np.savez_compressed(os.path.join(HERE, case["name"] + ".npz"), **d)
        print("wrote", case["name"], d["psi"].shape, d["rabi"].shape)
    for case in NUM_CASES:
        with tempfile.TemporaryDirectory() as tmp:
            d = make_numerical(case, tmp)
        np.savez_compressed(os.path.join(HERE, case["name"] + ".npz"), **d)
        print("wrote", case["name"], d["psi"].shape, d["rabi"].shape)
    for case in SOB_CASES:
        with tempfile.TemporaryDirectory() as tmp:
            d = make_sob(case, tmp)
        np.savez_compressed(os.path.join(HERE, case["name"] + ".npz"), **d)
        print("wrote", case["name"], "iterations", d["iterations"])


if __name__ == "__main__":
    main()
