"""Work partitioning over ranks (one process per GPU) and the gather of results.

The path shards without exchange: each pixel's samples and each job are independent. A frame is
split into contiguous row bands and a job list into per-rank shares balanced by work; the one
collective is the final gather of images to the destination rank (torch.distributed: NCCL
between GPUs, gloo on CPU). A row band keeps every pixel's sample order, so the assembled frame
equals a one-GPU render bit for bit (mr_render_rows).
"""

from __future__ import annotations

import numpy as np


def row_bands(height: int, world: int) -> list[tuple[int, int]]:
    """Contiguous row ranges [begin, end) covering [0, height), sizes differing by at most one."""
    if height < 0 or world < 1:
        raise ValueError("height must be >= 0 and world >= 1")
    base, extra = divmod(height, world)
    bands, begin = [], 0
    for rank in range(world):
        end = begin + base + (1 if rank < extra else 0)
        bands.append((begin, end))
        begin = end
    return bands


def job_cost(render, integrator) -> int:
    """Work estimate of a job: camera samples times the bounces a path may take."""
    depth = integrator.maximum_depth if integrator is not None else 8
    return render.width * render.height * render.samples_per_pixel * (depth + 1)


def partition_jobs(costs, world: int) -> list[list[int]]:
    """Longest-processing-time-first assignment of job indices to ranks (deterministic: ties go
    to the lower job index and the lower rank). Each rank's list is in job order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    loads = [0] * world
    shares: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        rank = min(range(world), key=lambda r: (loads[r], r))
        loads[rank] += costs[i]
        shares[rank].append(i)
    return [sorted(s) for s in shares]


def _dist():
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        raise RuntimeError("torch.distributed is not initialised")
    return dist


def gather_rows(band: np.ndarray, height: int, width: int, group=None, dst: int = 0):
    """Gathers every rank's row band (its rows of row_bands(height, world)) into the full
    (height, width, 3) image on `dst`; other ranks receive None."""
    import torch
    dist = _dist()
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    bands = row_bands(height, world)
    rows = max(e - b for b, e in bands)
    device = torch.device("cuda", torch.cuda.current_device()) \
        if dist.get_backend(group) == "nccl" else torch.device("cpu")
    begin, end = bands[rank]
    if band.shape != (end - begin, width, 3):
        raise ValueError(f"rank {rank} band has shape {band.shape}, expected {(end - begin, width, 3)}")
    padded = torch.zeros((rows, width, 3), dtype=torch.float32, device=device)
    if end > begin:
        padded[: end - begin] = torch.from_numpy(np.ascontiguousarray(band, np.float32)).to(device)
    parts = [torch.empty_like(padded) for _ in range(world)] if rank == dst else None
    dist.gather(padded, parts, dst=dst, group=group)
    if rank != dst:
        return None
    image = np.empty((height, width, 3), np.float32)
    for r, (b, e) in enumerate(bands):
        image[b:e] = parts[r][: e - b].cpu().numpy()
    return image


def render_frame_sharded(tracer, render, group=None, dst: int = 0, band_renderer=None):
    """PathTracer.render split into one row band per rank and gathered on `dst` (None on the
    other ranks). `band_renderer(render, begin, end)` defaults to tracer.render_rows."""
    dist = _dist()
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    begin, end = row_bands(render.height, world)[rank]
    renderer = band_renderer or (lambda r, b, e: tracer.render_rows(r, b, e))
    band = renderer(render, begin, end)
    return gather_rows(band, render.height, render.width, group, dst)


def render_jobs_sharded(jobs, group=None, dst: int = 0, batch_renderer=None, settings=None):
    """Renders a job list over the ranks: each rank takes its partition_jobs share, renders it
    with `batch_renderer(share_jobs)` (default: the batched engine) and the images are gathered
    on `dst` in job order (None on the other ranks)."""
    dist = _dist()
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    shares = partition_jobs([job_cost(j.render, j.integrator) for j in jobs], world)
    mine = shares[rank]
    if batch_renderer is None:
        from .api import render_batch

        def batch_renderer(share):
            images, _, _ = render_batch(share, settings)
            return images
    images = batch_renderer([jobs[i] for i in mine]) if mine else []
    gathered = [None] * world if rank == dst else None
    dist.gather_object(list(zip(mine, images)), gathered, dst=dst, group=group)
    if rank != dst:
        return None
    out = [None] * len(jobs)
    for part in gathered:
        for i, image in part:
            out[i] = image
    return out
