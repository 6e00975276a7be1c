"""ATUS-2's own programs built against the drop-in headers, against the
reference programs.

atus2_b200/host/bin holds rt_solver, bragg, double_bragg, bragg_ds, raman,
sobmin and gen_psi_0 compiled from ATUS-2's sources, unmodified, with the
drop-in CRT_Base / CRT_Base_IF / CRT_Base_IF_2 / CSOB_Base / cft_*d headers
(atus2_b200/dropin) and libatus_gpu.so.  The golden fixtures hold the XML
file and input .bin files the reference's own programs were run on, and what
they wrote.  The drop-in builds run the same files; their outputs must match
(FP64 bars of test_gpu_parity).  gen_psi_0 is host-only and is compared byte
for byte.  Without built programs (no ATUS-2 tree at build time) these tests
skip.
"""
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from atus2_b200 import binfmt
from golden_io import BRAGG_CASES, BRAGGDS_CASES, DBRAGG_CASES, NUM_CASES, RT_CASES, SOB_CASES, load
from gpu_util import rel_l2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "atus2_b200", "host", "bin")
REF = os.path.join(ROOT, "oracle", "_ref")


def run(prog, cwd, xml="run.xml", env=None):
    if not os.path.exists(os.path.join(BIN, prog)):
        pytest.skip(f"{prog} not built (needs the ATUS-2 source tree at build time)")
    e = dict(os.environ, MY_NO_OF_THREADS="4")
    e.update(env or {})
    r = subprocess.run([os.path.join(BIN, prog), xml], cwd=cwd, capture_output=True, text=True, env=e, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    return r.stdout


GEN_XML = """<SIMULATION>
  <DIM>{dim}</DIM>
  <FILENAME>inp.bin</FILENAME>
  <GUESS_{dim}D>{guess}</GUESS_{dim}D>
  <CONSTANTS><N>2.5</N><x0>0.5</x0><sx>1.5</sx></CONSTANTS>
  <ALGORITHM><NX>32</NX><NY>16</NY><NZ>8</NZ><XMIN>-8</XMIN><XMAX>8</XMAX><YMIN>-4</YMIN><YMAX>4</YMAX>
    <ZMIN>-2</ZMIN><ZMAX>2</ZMAX></ALGORITHM>
</SIMULATION>"""

GUESSES = {
    1: "exp(-0.5*(x-x0)^2/sx^2) + 0.2*rect(x,-1,1) - -x^2*1e-3",
    2: "exp(-0.5*((x-x0)^2/sx^2 + (y-1)^2)) * (1 + 0.3*rect(x,-1,1)*sign(y)) + Heaviside(x-2)*0.1",
    3: "exp(-(x*x+y*y+z*z)/2) * (x > 0 ? 1.5 : 1) + max(0, 1 - abs(z))",
}


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_gen_psi_0_byte_identical(dim):
    if not os.path.exists(os.path.join(REF, "gen_psi_0")):
        pytest.skip("reference programs not built")
    with tempfile.TemporaryDirectory() as tmp:
        open(os.path.join(tmp, "g.xml"), "w").write(GEN_XML.format(dim=dim, guess=GUESSES[dim]))
        # one thread each: the normalisation sum is an OpenMP reduction
        run("gen_psi_0", tmp, "g.xml", env={"OMP_NUM_THREADS": "1"})
        ours = open(os.path.join(tmp, "inp.bin"), "rb").read()
        r = subprocess.run([os.path.join(REF, "gen_psi_0"), "g.xml"], cwd=tmp, capture_output=True, timeout=120,
                           env=dict(os.environ, OMP_NUM_THREADS="1"))
        assert r.returncode == 0
        ref = open(os.path.join(tmp, "inp.bin"), "rb").read()
    assert ours == ref


def _write_inputs(g, tmp):
    xml = str(g["xml"])
    open(os.path.join(tmp, "run.xml"), "w").write(xml)
    if "psi0" in g:
        for c in range(g["psi0"].shape[0]):
            binfmt.write_bin(os.path.join(tmp, f"inp_{c + 1}.bin"), g["header"], g["psi0"][c])


def _outputs(tmp, ncomp):
    files = {}
    for fn in os.listdir(tmp):
        m = re.match(r"^(-?\d+\.\d{3})_(\d)\.bin$", fn)
        if m:
            files.setdefault(m.group(1), {})[int(m.group(2))] = fn
    out = []
    for key in sorted(files, key=float):
        recs = [binfmt.read_bin(os.path.join(tmp, files[key][c + 1])) for c in range(ncomp)]
        out.append((float(recs[0].header["t"]), np.stack([r.data for r in recs])))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name", RT_CASES + BRAGG_CASES + DBRAGG_CASES + BRAGGDS_CASES + NUM_CASES)
def test_realtime_program_matches_reference(name):
    _realtime_program(name)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["bragg2d", "dbragg1d", "braggds2d"])
def test_program_host_step_matches_reference(name):
    """The programs' own host bragg_ad (ATUS_HOST_STEPS=bragg_ad): the step
    runs on the host mirrors, the kinetic steps on the GPU -- the fallback
    path of any step function the drop-in has no kernel for."""
    _realtime_program(name, env={"ATUS_HOST_STEPS": "bragg_ad"})


def _realtime_program(name, env=None):
    from test_gpu_parity import FP64_TOL, state_close

    g = load(name)
    p = g["params"]
    prog = p["program"] if p["program"] in ("bragg", "double_bragg", "bragg_ds", "raman") else "rt_solver"

    def rabi_rows(path):
        return [[float(v) for v in ln.split()[1:]] for ln in open(path) if not ln.startswith("#") and ln.split()]

    with tempfile.TemporaryDirectory() as tmp:
        _write_inputs(g, tmp)
        run(prog, tmp, env=env)
        outs = _outputs(tmp, p["ncomp"])
        rabi = []
        for s in range(1, len(p["sequence"]) + 1):
            if prog == "bragg_ds":  # Spezie_<species>_Rabi_<seq>_<chirp>.txt, species side by side
                r1 = rabi_rows(os.path.join(tmp, f"Spezie_1_Rabi_{s}_0.txt"))
                r2 = rabi_rows(os.path.join(tmp, f"Spezie_2_Rabi_{s}_0.txt"))
                rabi += [a + b for a, b in zip(r1, r2)]
            elif prog != "rt_solver":
                rabi += rabi_rows(os.path.join(tmp, f"Rabi_{s}_0.txt"))
    assert len(outs) == len(g["t"])
    for (t, psi), t_ref, psi_ref in zip(outs, g["t"], g["psi"]):
        assert t == t_ref
        state_close(list(psi), list(psi_ref), FP64_TOL)
    if prog != "rt_solver":
        np.testing.assert_allclose(np.array(rabi), g["rabi"], rtol=5e-6, atol=1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["scan1d", "scan2d"])
@pytest.mark.parametrize("sequential", [False, True])
def test_phase_scan_matches_reference(name, sequential):
    """A phase scan (bragg_ad with no_of_chirps scans, chirp_mode 1) then
    freeprop, through ATUS-2's bragg program on the drop-in headers: scans
    1..n-1 side by side on clones of the context (default) or one after
    another (ATUS_SEQUENTIAL_SCANS=1); the .bin outputs (scan 0), the Rabi
    file of every scan and the Chirp file against the reference program."""
    from test_gpu_parity import FP64_TOL, state_close

    g = load(name)
    nc = int(g["params"]["chirps"])

    def rows(path):
        return np.array([[float(v) for v in ln.split()] for ln in open(path) if not ln.startswith("#") and ln.split()])

    with tempfile.TemporaryDirectory() as tmp:
        _write_inputs(g, tmp)
        run("bragg", tmp, env={"ATUS_SEQUENTIAL_SCANS": "1"} if sequential else None)
        outs = _outputs(tmp, 2)
        rabi = np.stack([rows(os.path.join(tmp, f"Rabi_1_{k}.txt")) for k in range(nc)])
        rabi_free = rows(os.path.join(tmp, "Rabi_2_0.txt"))
        chirp = rows(os.path.join(tmp, "Chirp_1.txt"))
    assert len(outs) == len(g["t"])
    for (t, psi), t_ref, psi_ref in zip(outs, g["t"], g["psi"]):
        assert t == t_ref
        state_close(list(psi), list(psi_ref), FP64_TOL)
    # six significant digits in the text files
    np.testing.assert_allclose(rabi, g["rabi_scans"], rtol=5e-6, atol=1e-10)
    np.testing.assert_allclose(rabi_free, g["rabi_free"], rtol=5e-6, atol=1e-10)
    np.testing.assert_allclose(chirp, g["chirp"], rtol=5e-6, atol=1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("name", SOB_CASES)
def test_sobmin_program_matches_reference(name):
    g = load(name)
    with tempfile.TemporaryDirectory() as tmp:
        _write_inputs(g, tmp)
        out = run("sobmin", tmp)
        final = binfmt.read_bin(os.path.join(tmp, "final.bin"))
        zero = binfmt.read_bin(os.path.join(tmp, "zero.bin"))
    iters = len(re.findall(r"^--- \d+$", out, re.M))
    assert abs(iters - int(g["iterations"])) <= 1
    assert rel_l2(final.data, g["psi"]) < 1e-10
    assert final.header.tobytes() == g["header"].tobytes()
    assert not zero.data.any()
