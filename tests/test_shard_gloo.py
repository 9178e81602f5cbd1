"""Sharding over ranks (hulktracer_b200/shard.py) with two gloo ranks on CPU:
frame sharding (disjoint frames covering the animation range, max / sum
reductions) and ray-tile sharding of one frame (row bands rendered per rank
-- here by the oracle, the GPU's restatement -- and gathered into the same
image one rank renders alone)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from hulktracer_b200.shard import frames_for_rank, gather_rows, reduce_job, rows_for_rank


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


def test_row_bands_cover_the_frame():
    for h in (1, 4, 7, 64, 720, 1081):
        for world in (1, 2, 3, 4, 8):
            bands = [rows_for_rank(h, r, world) for r in range(world)]
            assert bands[0][0] == 0 and bands[-1][1] == h
            for (a0, a1), (b0, b1) in zip(bands, bands[1:]):
                assert a1 == b0 and a0 <= a1
            for r, (y0, y1) in enumerate(bands[:-1]):
                assert y0 % 4 == 0 and (y1 - y0) % 4 == 0
    with pytest.raises(ValueError):
        rows_for_rank(10, 2, 2)


def band_worker(rank, world, port, q):
    import numpy as np
    import torch
    import torch.distributed as dist
    from hulktracer_b200 import scenes
    from oracle.oracle import NORM_IEEE, SHORTSTACK, Oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        W, H = 96, 70
        sc = scenes.static_small(width=W, height=H)
        O = Oracle()
        box = sc.scene_box()
        cn, cr = O.build_binned(sc.verts, sc.tris, box)
        tree = O.make_tree(sc.verts, sc.tris, O.cache(sc.verts, sc.tris, NORM_IEEE), O.compact_to_ref(cn), cr, box)
        rays = O.camera_rays(sc.camera, W, H, NORM_IEEE).reshape(H, W, 8)
        y0, y1 = rows_for_rank(H, rank, world)
        band = O.render_cpu(tree, np.ascontiguousarray(rays[y0:y1]).reshape(-1, 8), W, y1 - y0, sc.lights,
                            SHORTSTACK, 6, NORM_IEEE, nthreads=1)
        img = gather_rows(torch.from_numpy(band.view(np.int32).copy()), rank, world, W, H)
        full = O.render_cpu(tree, rays.reshape(-1, 8), W, H, sc.lights, SHORTSTACK, 6, NORM_IEEE, nthreads=1)
        q.put((rank, bool(np.array_equal(img.numpy().view(np.uint32), full)), int((full != 0).sum())))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_row_bands():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=band_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, equal, lit in res:
        assert equal and lit > 100
