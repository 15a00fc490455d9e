"""Multi-rank bench plumbing on CPU: two gloo ranks (127.0.0.1) agree on the
max-over-ranks step time and on the whole-job seconds per problem, and the
reference arm does no work on ranks other than 0."""
import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench.rank_barrier(dist, cuda=False)
        my_ms = 10.0 * (rank + 1)  # rank 1 is the slower replica
        t = bench.max_over_ranks_of(my_ms, dist, "cpu")
        v = bench.whole_job_seconds_per_problem(t / 4, world)  # 4 steps
        out[rank] = (t, v)
        bench.rank_barrier(dist, cuda=False)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_max_time_and_whole_job_value():
    world = 2
    out = mp.Manager().dict()
    mp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0] == out[1]
    t, v = out[0]
    assert t == pytest.approx(20.0)
    assert v == pytest.approx((20.0 / 4) / 1e3 / world)


def test_reference_arm_skips_non_zero_ranks(monkeypatch):
    import argparse

    import bench

    monkeypatch.setenv("RANK", "1")
    args = argparse.Namespace(warmup=1, steps=1, gpus=2)
    assert bench.run_reference(args) is None  # returns before touching the oracle


def test_single_process_paths_need_no_process_group():
    import bench

    assert bench.max_over_ranks_of(3.5, None, "cpu") == 3.5
    assert bench.whole_job_seconds_per_problem(56.0, 1) == pytest.approx(0.056)
