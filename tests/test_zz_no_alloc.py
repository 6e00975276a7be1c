"""atus_particle_number_noalloc, the entry point that allocates nothing,
called through the C ABI and checked against atus_particle_number on the
same fields: two calls in a row (a large field, then a small one, so that
partial sums left by the first call would spoil the second).  Collected
last; passes alone in a fresh process and after the other tests."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # the particle-number tolerance of the parity tests (another summation order)


def _solver(shape, prec, seed):
    from atus2_b200 import Solver, binfmt

    dim = len(shape)
    h = binfmt.make_header(dim, shape, [-8.0] * dim, [8.0] * dim)
    rng = np.random.default_rng(seed)
    s = Solver(h, 1, prec)
    psi = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    s.set_psi(0, psi)
    ar = float(np.prod([h[k] for k in ("dx", "dy", "dz")[:dim]]))
    return s, ar, int(np.prod(shape))


@pytest.mark.parametrize("prec_name", ["fp64", "mixed"])
def test_noalloc_particle_number_matches_context_reduction(prec_name):
    import torch

    from atus2_b200 import PREC_FP64, PREC_MIXED, engine

    prec = PREC_FP64 if prec_name == "fp64" else PREC_MIXED
    L = engine.load_library()
    out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
    cases = [_solver([128, 128, 64], prec, 1), _solver([256, 128], prec, 2)]
    for k, (s, ar, npts) in enumerate(cases):
        ref = s.particle_number(0)
        s.synchronize()
        rc = L.atus_particle_number_noalloc(C.c_void_p(s.device_ptr(0)), npts, prec, ar,
                                            C.c_void_p(out.data_ptr() + 8 * k), None)
        assert rc == 0
        torch.cuda.synchronize()
        got = float(out[k].item())
        assert got == pytest.approx(ref, rel=RTOL), (k, got, ref)


def test_noalloc_rejects_oversized_and_invalid_input():
    import torch

    from atus2_b200 import PREC_FP64, engine

    L = engine.load_library()
    buf = torch.zeros(4, dtype=torch.float64, device="cuda")
    p = C.c_void_p(buf.data_ptr())
    limit = 134217728  # ATUS_NOALLOC_MAX_POINTS
    assert L.atus_particle_number_noalloc(p, limit + 1, PREC_FP64, 1.0, p, None) == -6  # ATUS_E_LIMIT
    assert L.atus_particle_number_noalloc(p, 16, PREC_FP64, 1.0, None, None) == -1  # ATUS_E_ARG
    assert L.atus_particle_number_noalloc(p, 16, 7, 1.0, p, None) == -1
    torch.cuda.synchronize()
    assert float(buf.sum().item()) == 0.0  # nothing was launched
