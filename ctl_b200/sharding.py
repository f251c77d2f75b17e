"""Views across ranks: one process per GPU, the volume replicated on each.

Views are independent units (the reference round-robins them over OpenCL
devices with the volume replicated on each, raycasterprojector.cpp:321-357).
Here a rank takes one contiguous block of views, so its output is one
contiguous slice of [view][module][row][channel]; no data-path collective is
needed.  `gather_views` collects the slices on every rank when a consumer
needs the whole result in one place (torch.distributed, NCCL or gloo).
"""
from __future__ import annotations

from typing import Callable, Tuple

import numpy as np


def shard_views(n_views: int, world: int, rank: int) -> Tuple[int, int]:
    """[start, stop) of rank's views; sizes differ by at most one."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    base, extra = divmod(n_views, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def project_shard(project: Callable[[np.ndarray], object], pmats, world: int, rank: int):
    """Project this rank's views.  `project` maps a (views, modules, 3, 4) block of
    projection matrices to its projections (e.g. Context.project on a resident volume)."""
    start, stop = shard_views(int(pmats.shape[0]), world, rank)
    return start, stop, project(pmats[start:stop])


def broadcast_volume(volume, shape, src: int = 0, device=None, group=None):
    """The volume on every rank from rank `src` (the only rank that needs to read or
    generate it): one broadcast, over NVLink with NCCL on GPUs, in place of each rank
    loading its own copy (the reference uploads it to every device from the host,
    raycasterprojector.cpp:239-251).  `volume` is ignored on the other ranks."""
    import torch
    import torch.distributed as dist
    rank = dist.get_rank(group)
    if rank == src:
        t = torch.as_tensor(volume, dtype=torch.float32)
        t = t.to(device) if device is not None else t
        t = t.contiguous()
        if tuple(t.shape) != tuple(shape):
            raise ValueError(f"volume has shape {tuple(t.shape)}, expected {tuple(shape)}")
    else:
        t = torch.empty(tuple(shape), dtype=torch.float32, device=device)
    dist.broadcast(t, src=src, group=group)
    return t


def gather_views(local, n_views: int, world: int, rank: int, group=None):
    """All-gather the per-rank view slices into the full [view][...] tensor."""
    import torch
    import torch.distributed as dist
    sizes = [shard_views(n_views, world, r) for r in range(world)]
    longest = max(stop - start for start, stop in sizes)
    t = torch.as_tensor(local)
    padded = torch.zeros((longest,) + tuple(t.shape[1:]), dtype=t.dtype, device=t.device)
    padded[: t.shape[0]] = t
    parts = [torch.empty_like(padded) for _ in range(world)]
    dist.all_gather(parts, padded, group=group)
    return torch.cat([p[: stop - start] for p, (start, stop) in zip(parts, sizes)], dim=0)
