"""The multi-rank host logic of bench.py on CPU ranks (gloo, world size 2):
every rank learns the slowest rank's time, the whole-job rate counts every
rank's replica, and the reference arm runs on rank 0 alone."""
import io
import json
import os
import socket
import sys
from contextlib import redirect_stdout

import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world)
    try:
        ms = bench.max_over_ranks(1.0 + 2.0 * rank, dist, device="cpu")
        out[rank] = (ms, bench.job_rate(world, 10, 1000.0, ms))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_time_is_the_slowest_ranks_and_rate_counts_every_replica():
    world, port = 2, _free_port()
    out = mp.Manager().dict()
    mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
    for r in range(world):
        ms, rate = out[r]
        assert ms == 3.0
        assert abs(rate - 2 * 10 * 1000.0 / 3e-3) < 1e-6 * rate


def test_single_rank_needs_no_collective():
    assert bench.max_over_ranks(4.5, None) == 4.5
    assert bench.job_rate(1, 20, 16.0, 2.0) == 20 * 16.0 / 2e-3


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    args = bench.parse()
    buf = io.StringIO()
    with redirect_stdout(buf):
        assert bench.run_reference(args) == 0
    assert buf.getvalue() == ""  # no work, no line: rank 0 prints the job's line
