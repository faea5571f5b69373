"""bench.py's multi-rank host logic on CPU ranks over gloo (world size 2, 127.0.0.1): the slowest rank
sets the whole job's time, the whole-job rate counts every rank's cells, and the reference arm runs on
rank 0 alone (the other ranks return without work or output)."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        ms = 10.0 + 5.0 * rank                      # rank 1 is the slower one
        got = bench.allmax(dist, ms)
        rate = bench.whole_job_rate(dist, 1000, 4, world, ms)
        buf = io.StringIO()
        if rank != 0:
            class A:
                workload, steps, warmup = "riemann2000", 1, 0
            with redirect_stdout(buf):
                bench.run_reference(A(), rank, world)
        out.put((rank, got, rate, buf.getvalue()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, rate, printed in res:
        assert got == 15.0                          # the slowest rank's time
        assert rate == pytest.approx(1000 * 4 * 2 / 15e-3)
        if rank == 1:
            assert printed == ""                    # the reference arm's other ranks do nothing
