"""The multi-GPU path is replicas (frames and streams are independent): each
rank processes its own frames and the job's throughput is every rank's units
over the slowest rank's time. Checked here with two gloo ranks on the CPU,
through the same helpers bench.py uses under torchrun."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import datetime
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # Rank r took (1 + r) seconds for its 100 units.
        rate = bench.whole_job_rate(100.0, 1.0 + rank, world, dist, device="cpu")
        slowest = bench.max_over_ranks(1.0 + rank, dist, device="cpu")
        out[rank] = (rate, slowest)
    finally:
        dist.destroy_process_group()


def test_whole_job_rate_over_two_gloo_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        got = dict(out)
    # 2 ranks x 100 units over the slower rank's 2 s, the same on every rank.
    assert got == {0: (100.0, 2.0), 1: (100.0, 2.0)}


def test_single_rank_needs_no_process_group():
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    assert bench.whole_job_rate(50.0, 2.0, 1, None, device="cpu") == 25.0
