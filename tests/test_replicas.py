"""The N-GPU path of bench.py is replicas only: each rank times its own scene,
the job time is the max over ranks, and the value counts every rank's work.
Checked here with two gloo ranks on CPU (the reduction bench.py runs over
NCCL on GPUs)."""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 100.0 + 50.0 * rank  # rank 1 is the slower replica
        job_ms = bench.max_over_ranks(torch, dist, ms, torch.device("cpu"))
        q.put((rank, job_ms, bench.replica_value(1000, 10, world, job_ms)))
    finally:
        dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [150.0, 150.0]
    # 2 replicas x 1000 units x 10 steps in 0.15 s
    assert out[0][2] == pytest.approx(2 * 1000 * 10 / 0.15)


def test_single_rank_needs_no_collective():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(torch, None, 12.5, torch.device("cpu")) == 12.5
    assert bench.replica_value(128000, 200, 1, 84.8) == pytest.approx(128000 * 200 / 0.0848)
