"""The replicas path on CPU: two gloo ranks each build their own network (their own seed) and reduce their
timings the way bench.py does -- the max of the times, the sum of the work."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from naer2_b200.networks import brunel

        net, _ = brunel.build(**brunel.CONFIG0, seed=1 + rank)
        v0 = float(net.populations[0].V.sum())
        times = [10.0 + rank, 1.0 * (2 - rank)]
        counts = [100 * (rank + 1), 7]
        res = bench.reduce_over_ranks(times, counts, world, torch.device("cpu"))
        out[rank] = (res, v0)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_like_the_bench():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    (r0, v0), (r1, v1) = out[0], out[1]
    assert r0 == r1 == [11.0, 2.0, 300.0, 14.0]
    assert v0 != v1  # each replica its own seed
