"""The C-ABI library loads without a GPU and exports every entry point that
include/atus_gpu.h declares (no compute calls here)."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "atus_gpu.h")


def declared():
    return sorted(set(re.findall(r"ATUS_API [^;]*?\b(atus_\w+)\(", open(HEADER).read())))


def test_library_exports_header_symbols():
    from atus2_b200 import engine

    L = engine.load_library()
    for name in declared():
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", engine.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (atus_\w+)$", out, re.M))
    assert set(declared()) == exported


def test_binding_covers_header():
    from atus2_b200 import engine

    assert sorted(engine.SIGNATURES) == declared()


def test_no_device_means_error_not_fallback():
    """Creating a context without a usable device fails loudly."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import numpy as np

    from atus2_b200 import AtusError, Solver, binfmt

    h = binfmt.make_header(1, [64], [-1.0], [1.0])
    with pytest.raises(AtusError):
        Solver(h, 1)
