"""Multi-GPU plumbing on CPU: independent replicas under torch.distributed (gloo, two ranks).

Jobs never exchange data, so N GPUs run N independent replicas; the only
collective is the timing reduction: the job takes as long as the slowest rank
and the RIRs of every rank count (bench.replica_throughput).
"""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out) -> None:
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        local_ms = [12.0, 15.0][rank]
        ms, value = bench.replica_throughput(local_ms, 8, dist, "cpu")
        out.put((rank, ms, value))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks_and_counts_every_rank():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, value in results:
        assert ms == pytest.approx(15.0)
        assert value == pytest.approx(2 * 8 / 0.015)


def test_single_process_needs_no_collective():
    import bench
    ms, value = bench.replica_throughput(10.0, 8)
    assert ms == 10.0 and value == pytest.approx(800.0)
