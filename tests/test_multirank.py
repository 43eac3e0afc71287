"""The multi-GPU path of the bench on CPU ranks (gloo, world size 2).

The engine shards nothing: with N GPUs each rank steps its own replica of
the model, and the job's value counts the cell updates of all ranks over
the slowest rank's time. These tests run that protocol (barrier, the
max-over-ranks time, the aggregate) on two gloo processes, with a rank that
is slower than the other, and a rank that fails before the collective."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out, fail_rank):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    try:
        if rank == fail_rank:
            raise SystemExit(3)  # leaves before the collective: the others must not hang
        dist.barrier()
        t = bench.max_over_ranks(times[rank], world, "cpu")
        out[rank] = (t, bench.aggregate(world, 1000, 10, t))
    finally:
        if rank != fail_rank:
            dist.destroy_process_group()


def test_max_over_ranks_and_aggregate_on_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    times = [0.5, 2.0]
    mp.start_processes(_rank, args=(2, _port(), times, out, -1), nprocs=2, join=True, start_method="spawn")
    for r in range(2):
        t, v = out[r]
        assert t == 2.0                                  # the slowest rank's time
        assert v == pytest.approx(2 * 1000 * 10 / 2.0 / 1e6)


def test_a_rank_that_leaves_ends_the_job_with_an_error():
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    with pytest.raises(Exception):
        mp.start_processes(_rank, args=(2, _port(), [1.0, 1.0], out, 1), nprocs=2, join=True,
                           start_method="spawn")
    assert 0 not in out  # rank 0 got no result from a collective its peer never joined
