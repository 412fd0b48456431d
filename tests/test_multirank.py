"""The benchmark's multi-rank host logic on two CPU ranks (gloo): every rank
takes part in the max-over-ranks reduction of its device time and gets the
slowest rank's time back, the whole-job rate counts the units of all ranks
over that time, and on ranks other than 0 the reference arm returns
without work or output.  The device parts of the arms need a GPU; the N > 1
path is replicas (one independent subdomain per GPU), so these reductions
are its only exchange.
"""
import datetime
import io
import os
import socket
import sys
import types
from contextlib import redirect_stdout

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms_local = 10.0 * (rank + 1)                     # rank 1 is the slower one
        ms = bench.max_over_ranks(ms_local, dist, "cpu")
        rate = bench.whole_job_rate(1000, 4, world, ms)
        dist.barrier()
        q.put((rank, ms, rate))
    finally:
        dist.destroy_process_group()


def test_two_ranks_reduce_to_the_slowest():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0], codes
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, rate in got:
        assert ms == 20.0, (rank, ms)
        assert rate == pytest.approx(1000 * 4 * 2 / 0.020), (rank, rate)


def test_reference_arm_runs_on_rank_zero_only():
    sys.path.insert(0, ROOT)
    import bench
    args = types.SimpleNamespace(steps=1, warmup=3, gpus=2, workload="torus")
    out = io.StringIO()
    with redirect_stdout(out):
        bench.reference_arm(args, bench.WORKLOADS["torus"], 1)
    assert out.getvalue() == ""
