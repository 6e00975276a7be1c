"""Builds libatus_gpu.so in-tree for sm_100a.

    python -m atus2_b200.build [--jobs N]

Each csrc/*.cu file is compiled to an object with
``nvcc -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo`` (in parallel),
and the objects are linked into ``atus2_b200/libatus_gpu.so``.  Objects are
cached in ``atus2_b200/_build`` and rebuilt when a source or header changes.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libatus_gpu.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "-I", INCLUDE, "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: libatus_gpu.so cannot be built")


def _headers_mtime() -> float:
    hs = glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
    hs += glob.glob(os.path.join(INCLUDE, "*.h"))
    return max(os.path.getmtime(h) for h in hs)


def _compile(src: str, obj: str) -> None:
    cmd = [nvcc(), *ARCH, *FLAGS, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}")


def build(jobs: int | None = None, force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr = _headers_mtime()
    todo = []
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr):
            todo.append((s, o))
    if todo:
        jobs = jobs or max(1, min(len(todo), os.cpu_count() or 1))
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            futs = [ex.submit(_compile, s, o) for s, o in todo]
            for f in cf.as_completed(futs):
                f.result()
        if verbose:
            print(f"compiled {len(todo)} file(s)")
    if todo or force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        tmp = LIB + ".tmp"
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


HOST = os.path.join(HERE, "host")
DROPIN = os.path.join(HERE, "dropin")
# The ATUS-2 programs, by their source path in the ATUS-2 tree, and the
# headers each one uses without including them (the real FFTW / muParser /
# GSL headers pulled them in): the same force-includes as the oracle recipe.
PROGRAMS = {
    "rt_solver": ("source/SOLVER/src/rt_solver.cpp", []),
    "bragg": ("source/interferometry/src/bragg.cpp", []),
    "double_bragg": ("source/interferometry/src/double_bragg.cpp", []),
    "bragg_ds": ("source/interferometry/src/bragg_ds.cpp", ["complex"]),
    "raman": ("source/interferometry/src/raman.cpp", []),
    "sobmin": ("source/SOLVER/src/sob_solver.cpp", []),
    "gen_psi_0": ("source/utils/src/gen_psi_0.cpp", []),
}


def build_programs(tree: str | None = None, verbose: bool = False) -> list[str]:
    """Compiles ATUS-2's own program sources, unmodified, from the source tree
    `tree` (default: $ATUS2_REFERENCE_TREE) against the drop-in headers
    (atus2_b200/dropin: CRT_Base, CRT_Base_IF, CRT_Base_IF_2, CSOB_Base,
    cft_*d, ParameterHandler, muParser, fftw3) and libatus_gpu.so, into
    host/bin (found at run time next to the package, rpath $ORIGIN/../..).
    Without a tree nothing is built and the list is empty."""
    tree = tree or os.environ.get("ATUS2_REFERENCE_TREE")
    if not tree or not os.path.isdir(os.path.join(tree, "source")):
        return []
    out = os.path.join(HOST, "bin")
    os.makedirs(out, exist_ok=True)
    deps = [LIB] + glob.glob(os.path.join(HOST, "*.h")) + glob.glob(os.path.join(DROPIN, "*.h"))
    deps.append(os.path.join(INCLUDE, "atus_gpu.h"))
    newest = max(os.path.getmtime(d) for d in deps)
    built = []
    for p, (rel, force) in PROGRAMS.items():
        src = os.path.join(tree, rel)
        exe = os.path.join(out, p)
        built.append(exe)
        if os.path.exists(exe) and os.path.getmtime(exe) >= max(newest, os.path.getmtime(src)):
            continue
        inc = [a for f in force for a in ("-include", f)]
        cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", *inc, "-I", DROPIN, "-I", INCLUDE, "-o", exe, src, "-L", HERE,
               "-l:libatus_gpu.so", "-Wl,-rpath,$ORIGIN/../.."]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"g++ failed on {p} ({rel}):\n{r.stdout}\n{r.stderr}")
        if verbose:
            print("built", exe)
    return built


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--programs", metavar="TREE", help="also build ATUS-2's programs from this source tree")
    args = ap.parse_args()
    print(build(args.jobs, args.force, verbose=True))
    if args.programs:
        build_programs(args.programs, verbose=True)
