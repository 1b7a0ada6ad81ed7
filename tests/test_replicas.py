"""The multi-GPU path is replicas (every rank renders its own frames, no data-path
collective): the timing collectives and the whole-job aggregation, run as two gloo
ranks on the CPU."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    # rank r took 100 + 50 r ms for 2 steps of 1000 paths
    value, max_ms = bench.whole_job(1000, 2, 100.0 + 50.0 * rank, world)
    bench.barrier(world)
    out[rank] = (value, max_ms)
    dist.destroy_process_group()


def test_whole_job_rate_uses_the_slowest_rank():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    slow = 100.0 + 50.0 * (world - 1)
    for r in range(world):
        value, max_ms = res[r]
        assert max_ms == slow
        assert value == pytest.approx(world * 1000 * 2 / (slow / 1000.0))


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    import bench

    monkeypatch.setenv("RANK", "1")
    args = type("A", (), {"steps": 1, "warmup": 1, "gpus": 2})()
    assert bench.run_reference(args) == 0
