"""The benchmark's multi-rank path on CPU: two gloo ranks agree on the slowest
rank's time, the whole-job throughput counts every replica, and the reference arm
runs on rank 0 only (the other ranks exit without work)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, values, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        out[rank] = bench.max_over_ranks(values[rank], "cpu", world)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    world = 2
    values = [3.25, 7.5]
    with mp.get_context("spawn").Manager() as m:  # no fork of this process
        out = m.dict()
        mp.start_processes(_rank, args=(world, _free_port(), values, out), nprocs=world,
                           join=True, start_method="spawn")
        assert dict(out) == {0: 7.5, 1: 7.5}


def test_single_rank_and_throughput():
    assert bench.max_over_ranks(4.0, "cpu", 1) == 4.0
    # two replicas of 1000 DoFs, 5 steps in 10 ms: 1e6 DoF/s
    assert bench.replica_throughput(2, 1000, 5, 10.0) == pytest.approx(1e6)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    monkeypatch.setenv("RANK", "1")

    class Args:
        cpu_cells, warmup, steps, gpus = 8, 3, 1, 2
    assert bench.run_reference(Args()) == 0
    assert capsys.readouterr().out == ""


def test_reference_arm_bounds_its_sample_and_keeps_the_config(monkeypatch, capsys):
    """The CPU reference arm on rank 0 times at most REF_STEPS steps after at most REF_WARMUP,
    says so, and prints the GPU arm's config for the same mesh."""
    import json
    monkeypatch.setenv("RANK", "0")

    class Args:
        cpu_cells, warmup, steps, gpus = 6, 5, 20, 1
    assert bench.run_reference(Args()) == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["steps"] == bench.REF_STEPS and line["warmup"] == bench.REF_WARMUP
    assert line["steps_requested"] == 20 and line["warmup_requested"] == 5
    assert line["config"] == bench.workload_config(6)
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] == "port"


def test_cpu_sample_keeps_the_first_step():
    keep = {}
    rate, sec, n, cores = bench.cpu_step_sample(4, 1, keep=keep)
    assert keep["T1"].shape == (n,) and rate > 0
    assert keep["T1"].max() > 0.0  # the source heated the first step
