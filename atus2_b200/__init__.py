"""B200-native engine for ATUS-2's split-step Fourier Gross-Pitaevskii path.

The compute path is ``libatus_gpu.so`` (hand-written sm_100a kernels behind the
C ABI of include/atus_gpu.h); ``engine.Solver`` binds it with ctypes and
``binfmt`` reads and writes the reference's ``.bin`` files.
"""
from . import binfmt  # noqa: F401
from .engine import (  # noqa: F401
    PREC_FP64,
    PREC_MIXED,
    STEP_BRAGG_AD,
    STEP_DOUBLE_BRAGG_AD,
    STEP_NL_IF_2,
    STEP_BRAGG_DS_AD,
    STEP_NUMERICAL_BRAGG,
    STEP_NUMERICAL_RAMAN,
    STEP_NL,
    STEP_NL_IF,
    AtusError,
    Batch,
    Laser,
    Solver,
    load_library,
)
