"""The multi-rank bench path on CPU: two ``gloo`` ranks (spawned processes).

``bench.py --gpus N`` under torchrun runs one independent replica per rank; the only
exchange is the max over ranks of the timed region, and ``value`` counts every rank's
matvecs over that slowest time.  The reference arm runs on rank 0 alone.  These are the
host-side pieces of that path; the ranks here are CPU processes.
"""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        ms = bench.max_over_ranks(10.0 * (rank + 1), "cpu")  # rank r timed 10 (r + 1) ms
        out[rank] = (ms, bench.job_value(1_000_000, 4, world, ms))
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time_and_count_every_rank():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == 20.0
    # 2 ranks x 4 matvecs x 1 MFLOP in 20 ms
    assert res[0][1] == pytest.approx(2 * 4 * 1e6 / 20e-3 / 1e12)


def test_single_process_keeps_its_time():
    import bench

    assert not dist.is_initialized()
    assert bench.max_over_ranks(3.5, "cpu") == 3.5


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    """Under torchrun every rank starts the reference arm; ranks other than 0 exit at once
    with no work and no output."""
    import argparse

    import bench

    monkeypatch.setitem(os.environ, "RANK", "1")
    bench.run_reference(argparse.Namespace(gpus=2, steps=3, warmup=3, cpu_budget=1.0))
    assert capsys.readouterr().out == ""
