"""The bench's multi-rank aggregation, run as two gloo ranks on the CPU."""

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = 100.0 + 50.0 * rank  # rank 1 is the slow one
        total = bench.max_over_ranks(local_ms, dist)
        q.put((rank, total, bench.whole_job_rate(10, world, total)))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_max_over_ranks_and_whole_job_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    for rank, total, rate in out:
        assert total == 150.0  # both ranks see the slowest rank's time
        assert rate == pytest.approx(2 * 10 / 0.150)


def test_single_rank_is_local():
    assert bench.max_over_ranks(12.5) == 12.5
    assert bench.whole_job_rate(300, 1, 750.0) == pytest.approx(400.0)
