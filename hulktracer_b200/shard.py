"""Frame sharding across ranks (one process per GPU) with no data-path
collective: rank r renders frames first + r, first + r + N, ... of the
animation, each on its own replica of the scene and tree. The only
collectives are the timing ones: the job's time is the maximum over ranks and
its work the sum, so throughput = total units / max time.
"""
from __future__ import annotations


def frames_for_rank(first: int, steps: int, rank: int, world: int) -> list[int]:
    """The `steps` frames rank `rank` of `world` renders, starting at frame `first`."""
    if world < 1 or not 0 <= rank < world or steps < 0:
        raise ValueError("bad rank / world / steps")
    return [first + rank + world * i for i in range(steps)]


def reduce_job(times, units, world: int, device="cpu"):
    """(max over ranks of each time, sum over ranks of `units`) through
    torch.distributed (any initialised backend; `device` must suit it:
    "cuda" for NCCL, "cpu" for gloo). With world == 1 it returns the inputs."""
    times = [float(t) for t in times]
    if world == 1:
        return times, float(units)
    import torch
    import torch.distributed as dist
    t = torch.tensor(times, dtype=torch.float64, device=device)
    u = torch.tensor([float(units)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return [float(x) for x in t.cpu()], float(u.cpu()[0])
