"""Frame sharding over ranks (hulktracer_b200/shard.py) with two gloo ranks on
CPU: the ranks' frames are disjoint and cover the animation range, and the
job time / work reductions are max / sum over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from hulktracer_b200.shard import frames_for_rank, reduce_job


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        frames = frames_for_rank(5, 7, rank, world)
        got = [None] * world
        dist.all_gather_object(got, frames)
        times, units = reduce_job([1.0 + rank, 10.0 - rank], 100 * (rank + 1), world)
        q.put((rank, got, times, units))
    finally:
        dist.destroy_process_group()


def test_frames_single_rank():
    assert frames_for_rank(3, 4, 0, 1) == [3, 4, 5, 6]
    with pytest.raises(ValueError):
        frames_for_rank(0, 1, 2, 2)
    assert reduce_job([1.5], 7, 1) == ([1.5], 7.0)


def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, times, units in res:
        flat = sorted(f for fr in got for f in fr)
        assert flat == list(range(5, 5 + 7 * world))
        assert not set(got[0]) & set(got[1])
        assert times == [2.0, 10.0]
        assert units == 300.0
