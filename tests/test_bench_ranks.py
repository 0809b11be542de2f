"""The bench's whole-job aggregation over ranks (units summed, time = the
slowest rank), run as two gloo processes on the CPU: the same collectives
bench.py issues over NCCL under torchrun."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        units, ms = bench.job_totals(100.0 + rank, 10.0 * (rank + 1), world, "cpu")
        q.put((rank, units, ms))
    finally:
        dist.destroy_process_group()


def test_job_totals_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, units, ms in got:
        assert units == 201.0  # 100 + 101
        assert ms == 20.0      # the slower rank


def test_job_totals_single_rank_is_identity():
    import bench

    assert bench.job_totals(5.0, 2.0, 1, "cpu") == (5.0, 2.0)
