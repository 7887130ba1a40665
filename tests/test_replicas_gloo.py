"""The replicas path of bench.py (--gpus N > 1: one independent replica per
rank, whole-job time = the slowest rank's) on CPU ranks over gloo."""

from __future__ import annotations

import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as tmp  # noqa: E402


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    import datetime
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r timed (10 + r) ms for the FP32 arm and (30 - r) ms for the FP64 arm
        got = bench.max_over_ranks([10.0 + rank, 30.0 - rank], world, "cpu")
        out.put((rank, got))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_max_over_ranks_takes_the_slowest_rank(world):
    ctx = tmp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = dict(out.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(world):
        assert results[r] == [10.0 + world - 1, 30.0]


def test_single_rank_is_the_identity():
    import bench

    assert bench.max_over_ranks([1.5, 2.5], 1, "cpu") == [1.5, 2.5]
