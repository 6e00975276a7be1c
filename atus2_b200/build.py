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
    build_programs(verbose=verbose)
    return LIB


HOST = os.path.join(HERE, "host")
PROGRAMS = ("rt_solver", "bragg", "double_bragg", "bragg_ds", "raman", "sobmin", "gen_psi_0")


def build_programs(verbose: bool = False) -> None:
    """The XML programs (host/programs/*.cpp) linked against libatus_gpu.so,
    found at run time next to the package (rpath $ORIGIN/../..)."""
    out = os.path.join(HOST, "bin")
    os.makedirs(out, exist_ok=True)
    deps = [LIB] + glob.glob(os.path.join(HOST, "*.h")) + [os.path.join(INCLUDE, "atus_gpu.h")]
    newest = max(os.path.getmtime(d) for d in deps)
    for p in PROGRAMS:
        src = os.path.join(HOST, "programs", p + ".cpp")
        exe = os.path.join(out, p)
        if os.path.exists(exe) and os.path.getmtime(exe) >= max(newest, os.path.getmtime(src)):
            continue
        cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-I", INCLUDE, "-o", exe, src, "-L", HERE,
               "-l:libatus_gpu.so", "-Wl,-rpath,$ORIGIN/../.."]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"g++ failed on {p}:\n{r.stdout}\n{r.stderr}")
        if verbose:
            print("built", exe)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    print(build(args.jobs, args.force, verbose=True))
