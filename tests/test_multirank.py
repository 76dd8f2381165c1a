"""Multi-rank host logic of bench.py on CPU (gloo, world size 2): the
max-over-ranks device time, the whole-job rate, and the reference arm's
"rank 0 only" behaviour. The data path has no collective (replicas only)."""
import multiprocessing as mp
import os
import socket
import sys
from datetime import timedelta

import pytest

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist)
        rate = bench.whole_job_rate(world, 8, ms)
        dist.barrier()
        q.put((rank, ms, rate))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_rate_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, rate in got:
        assert ms == 15.0                      # the slowest rank's time on every rank
        assert rate == pytest.approx(2 * 8 / 0.015)


def test_single_process_helpers():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.whole_job_rate(1, 10, 2.0) == pytest.approx(5000.0)


def test_reference_arm_nonzero_rank_exits_without_work(monkeypatch, capsys):
    sys.path.insert(0, str(ROOT))
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--steps", "2", "--warmup", "3"])
    assert bench.main() == 0
    assert capsys.readouterr().out == ""
