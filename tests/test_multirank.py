"""The N > 1 path of bench.py on the CPU: two ranks over gloo (127.0.0.1).

SHGEMM has no cross-GPU exchange, so `bench.py --gpus N` runs N replicas; the only
collective is the max-over-ranks reduction of each timed region, and the reference arm
runs on rank 0 alone. Both are exercised here with world_size 2 and no GPU.
"""
import json
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        ms = bench.max_over_ranks(local_ms, dist, "cpu")
        value = bench.aggregate_tflops(world, 1e12, ms)
        dist.barrier()
    finally:
        dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"ms": ms, "value": value}, f)


def test_two_ranks_take_the_slowest_time(tmp_path):
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    res = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(world)]
    for r in res:
        assert r["ms"] == 15.0  # max over ranks, seen identically by every rank
        assert abs(r["value"] - 2 * 1e12 / 0.015 / 1e12) < 1e-9  # both replicas' work over the slowest time


def test_single_rank_helpers_need_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert abs(bench.aggregate_tflops(1, 2e12, 1000.0) - 2.0) < 1e-12


def test_reference_arm_other_ranks_exit_without_output(capsys, monkeypatch):
    """Under torchrun the reference arm runs on rank 0 only; rank 1 returns 0 and prints nothing."""
    sys.path.insert(0, ROOT)
    import argparse

    import bench

    monkeypatch.setenv("RANK", "1")
    args = argparse.Namespace(steps=1, warmup=3, gpus=2, workload="square16k")
    assert bench.run_reference_arm(args, bench.WORKLOADS["square16k"]) == 0
    assert capsys.readouterr().out == ""
