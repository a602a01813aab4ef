"""The bench's multi-rank plumbing on CPU: two gloo ranks, as torchrun starts
them, meet at the barrier, agree on the max of their timings, and report the
whole-job rate; the reference arm does its work on rank 0 only."""
from __future__ import annotations

import importlib.util
import os
import socket

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    bench = _bench()
    r, w, dist = bench.dist_setup(world, backend="gloo")
    try:
        bench.barrier(dist)
        ms = 1000.0 + 250.0 * r   # the ranks' own timings differ
        total = bench.max_over_ranks(ms, dist)
        rate = bench.aggregate_rate(w, 1920 * 1080 * 256, 3, total)
        bench.barrier(dist)
        q.put((r, w, total, rate))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_rank():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0]
    out = sorted(q.get(timeout=5) for _ in range(world))
    slowest = 1000.0 + 250.0 * (world - 1)
    for r, w, total, rate in out:
        assert w == world and total == slowest
        assert rate == pytest.approx(world * 1920 * 1080 * 256 * 3 / (slowest / 1e3) / 1e6)


def test_single_process_needs_no_process_group(monkeypatch):
    monkeypatch.setenv("WORLD_SIZE", "1")
    bench = _bench()
    assert bench.dist_setup(1) == (0, 1, None)
    assert bench.max_over_ranks(3.5, None) == 3.5
    assert bench.aggregate_rate(1, 2e6, 2, 1000.0) == pytest.approx(4.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    """Under torchrun, ranks other than 0 leave the reference arm at once."""
    monkeypatch.setenv("RANK", "1")
    bench = _bench()

    class Args:
        gpus, steps, warmup = 2, 1, 0

    assert bench.run_reference(Args()) is None
