"""Work split across ranks (one process per GPU).

* Frame sharding, no data-path collective: rank r renders frames first + r,
  first + r + N, ... of the animation, each on its own replica of the scene
  and tree. The only collectives are the timing ones: the job's time is the
  maximum over ranks and its work the sum, so throughput = total units / max
  time.
* Ray-tile sharding of one frame: every rank builds the frame's tree on its
  own replica of the scene (the build is replicated rather than broadcast)
  and renders one contiguous band of rows (hk_render_rows_device, bands in
  multiples of 4 rows so the 8 x 4 ray tiles stay whole); the framebuffer is
  then gathered over the process group (NCCL over NVLink on GPUs) with one
  all_gather. No multicast.
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


def rows_for_rank(height: int, rank: int, world: int, align: int = 4) -> tuple[int, int]:
    """Row band [y0, y1) of `rank`: contiguous bands covering 0 .. height, each
    a multiple of `align` rows except the last, which also takes the rows
    past the last multiple of `align`."""
    if world < 1 or not 0 <= rank < world or height < 1 or align < 1:
        raise ValueError("bad rank / world / height")
    units = height // align
    base, extra = divmod(units, world)
    y0 = align * (rank * base + min(rank, extra))
    y1 = y0 + align * (base + (1 if rank < extra else 0))
    if rank == world - 1:
        y1 = height
    return y0, y1


def gather_rows(band, rank: int, world: int, width: int, height: int, align: int = 4):
    """The whole width x height image on every rank from each rank's band
    (a 1-D tensor of width x (y1 - y0) pixels, rows_for_rank's split): one
    all_gather of equal-sized buffers (bands padded to the largest)."""
    if world == 1:
        return band
    import torch
    import torch.distributed as dist
    bands = [rows_for_rank(height, r, world, align) for r in range(world)]
    y0, y1 = bands[rank]
    if band.numel() != (y1 - y0) * width:
        raise ValueError("band size does not match rows_for_rank")
    maxn = max((b1 - b0) * width for b0, b1 in bands)
    buf = torch.zeros(maxn, dtype=band.dtype, device=band.device)
    buf[: band.numel()] = band
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    return torch.cat([parts[r][: (b1 - b0) * width] for r, (b0, b1) in enumerate(bands)])
