"""The benchmark's multi-GPU logic (independent replicas, slowest rank's time,
whole-job throughput) with world-size-2 gloo ranks on CPU."""

from __future__ import annotations

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


def _rank(rank: int, world: int, port: int, results) -> None:
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        # Rank r pretends its steps took (10 + r) ms and (3 + 2 r) ms.
        total, other = bench.max_over_ranks([10.0 * (1 + rank), 3.0 + 2 * rank])
        results[rank] = (total, other, bench.replica_throughput(world, 1000, total, 10))
    finally:
        dist.destroy_process_group()


def test_ranks_agree_on_the_slowest_time_and_the_job_throughput():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    results = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, results)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert results[0] == results[1]
    total, other, value = results[0]
    assert total == 20.0 and other == 5.0
    # Two replicas of 1000 units, 10 steps in 20 ms: 2 x 1000 / 2 ms.
    assert value == pytest.approx(2 * 1000 / 2e-3)


def test_single_process_passes_values_through():
    import bench

    assert bench.max_over_ranks([1.5, 2.5]) == [1.5, 2.5]
    assert bench.replica_throughput(1, 100, 50.0, 5) == pytest.approx(100 / 0.01)
