"""The multi-GPU path of bench.py on CPU: two gloo ranks (replicas, no data
exchange) -- process-group set-up from the torchrun environment, the
max-over-ranks device time, the whole-job rate, and the reference arm, which
only rank 0 runs."""
import io
import contextlib
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(ws), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    r, w, local, dist = bench.dist_init()
    try:
        ms = 10.0 * (rank + 1)  # a slower rank 1
        ms_max = bench.max_over_ranks(dist, ms)
        rate = bench.whole_job_rate(w, 1000.0, ms_max)
        bench.barrier(dist)

        class Args:
            steps, warmup = 2, 3

        out = io.StringIO()
        ran = None
        if r != 0:  # the other ranks leave the reference arm without work or output
            with contextlib.redirect_stdout(out):
                ran = bench.reference_arm(Args(), r, w, dist)
        q.put((r, w, ms_max, rate, out.getvalue(), ran))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_replicas_on_gloo():
    ws, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(ws))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, w, ms_max, rate, printed, ran in res:
        assert w == ws
        assert ms_max == 20.0                  # the slowest rank's time, on every rank
        assert rate == pytest.approx(2 * 1000.0 / 20e-3)  # all ranks' units over that time
    assert res[1][4] == "" and res[1][5] is None  # rank 1: no reference run, no JSON line
