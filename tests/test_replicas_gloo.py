"""The bench's replica timing across ranks, on the CPU with two gloo ranks.

Each rank of ``bench.py --gpus N`` runs its own hemispheres (replicas; the path
has no exchange step).  The job's figure is the slowest rank's timed total over
the hemispheres all ranks processed, the same on every rank; the reference arm
runs on rank 0 alone.
"""

from __future__ import annotations

import os
import socket
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, results) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        assert bench.dist_env() == (world, rank, rank)
        local_ms = [1200.0, 1500.0][rank]  # rank 1 is the slower replica
        steps = 5
        value = bench.job_seconds_per_unit(local_ms, steps, world, torch.device("cpu"))
        results[rank] = value
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_agree_on_the_slowest_replica():
    world = 2
    manager = mp.Manager()
    results = manager.dict()
    mp.spawn(_rank_main, args=(world, _free_port(), results), nprocs=world, join=True)
    expected = 1500.0 / 1e3 / (5 * world)  # max over ranks / hemispheres of the whole job
    assert results[0] == pytest.approx(expected, rel=0, abs=1e-15)
    assert results[1] == results[0]


def test_single_process_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.job_seconds_per_unit(2000.0, 4, 1, torch.device("cpu")) == pytest.approx(0.5)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, str(ROOT))
    import bench

    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("LOCAL_RANK", "1")
    args = bench.parse_args(["--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"])
    assert bench.run_reference(args) == 0  # returns before any work
    assert capsys.readouterr().out == ""


def test_reference_arm_line_follows_the_bench_contract(monkeypatch, capsys):
    """The reference arm's JSON line: the native arm's metric, unit, direction and workload
    config, a cpu_baseline describing the run, and an e2e entry with no device copies."""

    import json

    sys.path.insert(0, str(ROOT))
    import bench

    for name in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(name, raising=False)
    stages = {"stages_1_5": {"measured_s": 1.5, "fraction": 1.0, "scaled_s": 1.5},
              "sweeps": {"measured_s": 1.5, "fraction": 0.1, "scaled_s": 15.0}}

    class FakeSampler:
        cores = 3

        def __init__(self, meshes):
            pass

        def sample(self):
            return {"total": 140.0, "measured_s": 3.0, "stages": stages}

        def close(self):
            pass

    monkeypatch.setattr(bench, "CpuSampler", FakeSampler)
    args = bench.parse_args(["--impl", "reference", "--steps", "2", "--warmup", "1"])
    assert bench.run_reference(args) == 0
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert (line["metric"], line["unit"], line["higher_is_better"]) == (bench.METRIC, bench.UNIT, False)
    assert line["value"] == pytest.approx(140.0) and line["steps"] == 2 and line["warmup"] == 1
    # a step is the measured sample: the driver's wall clock covers steps x ms_per_step
    assert line["ms_per_step"] == pytest.approx(3000.0) and line["extrapolated"] is True
    config = dict(line["config"])
    assert config.pop("parallelism")
    assert config == json.loads(json.dumps(bench.workload_config(bench.load_meshes())))
    baseline = line["cpu_baseline"]
    assert baseline["value"] == line["value"] and baseline["kind"] == "port" and baseline["cores"] == 3
    assert baseline["sample"] and baseline["stages_s"] == stages
    assert line["e2e"] == {"value": line["value"], "unit": bench.UNIT, "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_batched_legs_shard_units_by_cost():
    """Every unit goes to exactly one rank; the ranks' total costs stay close."""

    sys.path.insert(0, str(ROOT))
    import bench

    costs = [55679, 68864, 72655, 74933, 81661, 93349, 103165, 106130, 106236, 111415, 112878, 122399, 135336,
             141626, 150137, 152628]
    assert bench.shard_by_cost(costs, 1, 0) == list(range(16))
    for world in (2, 3, 4, 8):
        shards = [bench.shard_by_cost(costs, world, r) for r in range(world)]
        assert sorted(i for s in shards for i in s) == list(range(16))
        totals = [sum(costs[i] for i in s) for s in shards]
        assert max(totals) - min(totals) <= max(costs)


def _throughput_main(rank: int, world: int, port: int, results) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        results[rank] = bench.job_throughput([7.0, 9.0][rank], [100.0, 250.0][rank], world, torch.device("cpu"))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_batched_leg_throughput_is_all_units_over_the_slowest_rank():
    world = 2
    manager = mp.Manager()
    results = manager.dict()
    mp.spawn(_throughput_main, args=(world, _free_port(), results), nprocs=world, join=True)
    assert results[0] == results[1] == (16.0, 250.0)
