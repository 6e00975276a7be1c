"""Bounded waits on the GPU: the strided 256-point passes wait on an mbarrier
for each TMA tile copy, at most a set number of try_wait rounds.  A copy that
never completes must end the call with an error status the host reads, not
hang the GPU.  The test makes every wait run out without any fault: the
kernel issues no tile copy and no arrival, so the barrier phase never
completes and nothing is in flight when the kernel returns."""
import os

import numpy as np
import pytest

from atus2_b200 import PREC_FP64, AtusError, Solver, binfmt
from replay import KIND_NL

pytestmark = pytest.mark.gpu


def _solver(h, psi, V):
    s = Solver(h, 1, PREC_FP64)
    s.set_psi(0, psi)
    s.set_alpha(0, [0.5, 0.5])
    s.set_gs([5.0])
    s.set_potential(0, V)
    s.set_dt(1e-3)
    return s


@pytest.mark.skipif(os.environ.get("ATUS_TMA") == "0", reason="TMA-fed passes switched off")
def test_tma_wait_runs_out_and_reports():
    """256 x 256 (the x pass is a strided 256-point pass): with the copies
    dropped and a bound of 1000 rounds the block returns ATUS_E_CUDA; with
    the defaults restored the same context then runs a block identical to a
    fresh context's."""
    h = binfmt.make_header(2, [256, 256], [-8.0, -8.0], [8.0, 8.0])
    x = binfmt.x_coords(h, 0)[:, None]
    y = binfmt.x_coords(h, 1)[None, :]
    psi = (np.exp(-0.5 * (x * x + y * y)) * np.exp(1j * x)).astype(np.complex128)
    V = 0.5 * (x * x + y * y) + 0 * y
    s = _solver(h, psi, V)
    s.set_wait_limits(1000, True)
    with pytest.raises(AtusError, match="TMA tile copy did not complete"):
        s.block(2, KIND_NL)
    s.set_wait_limits()
    s.set_psi(0, psi)
    s.t = 0.0
    s.block(5, KIND_NL)
    ref = _solver(h, psi, V)
    ref.block(5, KIND_NL)
    assert s.t == ref.t
    np.testing.assert_array_equal(s.psi(0), ref.psi(0))
    s.close()
    ref.close()
