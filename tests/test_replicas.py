"""The multi-GPU path of bench.py is "replicas only": every rank runs the whole
workload and the one collective is the max of the timed region over ranks.
These tests run that path as two gloo ranks on the CPU."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    import datetime

    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    t = bench.max_over_ranks(dist, times[rank], "cpu")
    t2 = bench.max_over_ranks(dist, 2.0 * times[rank], "cpu")  # same collective order on every rank
    out[rank] = (t, t2, bench.whole_job_rate(world, 3, t))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_whole_job_rate_two_gloo_ranks():
    import torch.multiprocessing as mp

    world, port = 2, _free_port()
    times = [1.25, 2.5]
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, times, out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        t, t2, rate = res[r]
        assert t == max(times) and t2 == 2.0 * max(times)
        assert rate == pytest.approx(world * 3 / max(times))


def test_single_rank_needs_no_collective():
    import bench

    assert bench.max_over_ranks(None, 1.5, "cpu") == 1.5
    assert bench.whole_job_rate(1, 4, 2.0) == 2.0
