"""The N > 1 bench path on CPU: two gloo ranks run the replica bookkeeping that
`bench.py --gpus 2` runs over NCCL (each rank times its own replica; the step
time is the slowest rank's; the whole-job rate counts every rank's rows), and
the reference arm prints from rank 0 only."""

import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, torch.device("cpu"), world)
        rate = bench.replica_rate(1_000_000, world, ms)
        buf = io.StringIO()

        class A:  # only the fields run_reference reads before returning on rank != 0
            workload = "groupby"
            steps = 1
            warmup = 0
        with redirect_stdout(buf):
            if rank != 0:
                bench.run_reference(A, rank, world)
        out[rank] = (ms, rate, buf.getvalue())
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_replica_bookkeeping():
    world = 2
    port = _free_port()
    out = mp.Manager().dict()
    mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
    assert out[0][0] == out[1][0] == pytest.approx(15.0)          # the slowest rank's time
    assert out[0][1] == out[1][1] == pytest.approx(2 * 1_000_000 / 0.015 / 1e6)
    assert out[1][2] == ""                                         # non-zero ranks print nothing
