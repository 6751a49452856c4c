"""The multi-GPU timing of bench.py (independent replicas, one process per GPU): every rank takes the
slowest rank's time through one MAX all-reduce, and the whole-job value is all ranks' units over that
time.  Run as two gloo ranks on the CPU (the same calls run over NCCL on GPUs)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
torch = pytest.importorskip("torch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 + 5.0 * rank  # rank 1 is the slower replica
        ms_max = bench.max_over_ranks(ms, world, "cpu")
        value = bench.replica_throughput(1_000_000, world, 4, ms_max * 1e-3)
        out[rank] = (ms_max, value)
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank_time():
    import torch.multiprocessing as mp

    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
    assert out[0] == out[1]
    ms_max, value = out[0]
    assert ms_max == 15.0
    # 2 ranks x 4 steps x 1e6 path samples in 15 ms
    assert value == pytest.approx(2 * 4 * 1_000_000 / 15e-3 / 1e6)


def test_one_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(7.5, 1, "cpu") == 7.5
    assert bench.replica_throughput(16_777_216, 1, 10, 0.3) == pytest.approx(559.24, rel=1e-4)
