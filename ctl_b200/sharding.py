"""Work across ranks: one process per GPU, volumes replicated.

Views are independent units (the reference round-robins them over OpenCL
devices with the volume replicated on each, raycasterprojector.cpp:321-357).
Here a rank takes one contiguous block of views, so its output is one
contiguous slice of [view][module][row][channel]; no data-path collective is
needed.  `gather_views` collects the slices on every rank when a consumer
needs the whole result in one place (torch.distributed, NCCL or gloo).

Batches of uneven requests are spread by their sample counts (`shard_batch`,
longest first), and serving requests are routed by volume to the least-loaded
rank that holds it (`Router`, `serve_on_ranks`).
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

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


# ---- batches of uneven requests --------------------------------------------------------------

def lpt_assign(costs: Sequence[float], world: int) -> List[int]:
    """Rank of each item under longest-processing-time-first: items in
    decreasing cost (ties by index) each go to the least-loaded rank (ties to
    the lowest rank).  The busiest rank's load is within 4/3 of the best
    possible (Graham's bound for LPT).  Deterministic, so every rank computes
    the same assignment from the same costs."""
    if world < 1:
        raise ValueError(f"bad world size {world}")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    out = [0] * len(costs)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[i] = r
        load[r] += float(costs[i])
    return out


def shard_batch(costs: Sequence[float], world: int, rank: int) -> List[int]:
    """Indices (in input order) of the requests of a batch that `rank` projects.
    Costs are the requests' sample counts (Context.count_samples gives the exact
    count of the reference scheme), so ranks get about equal work although the
    volumes, view counts and detectors differ."""
    if not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    return [i for i, r in enumerate(lpt_assign(costs, world)) if r == rank]


# ---- serving on several GPUs ------------------------------------------------------------------

def volume_homes(n_volumes: int, world: int, replicas: Optional[int] = None) -> List[List[int]]:
    """The ranks that hold each volume resident: all ranks (replicas None or
    >= world), else `replicas` consecutive ranks starting at volume % world."""
    k = world if replicas is None else max(1, min(int(replicas), world))
    return [sorted((v + j) % world for j in range(k)) for v in range(n_volumes)]


class Router:
    """Routes serving requests to ranks, one DRRServer per GPU.

    A request for volume v goes to the rank among v's homes with the least
    outstanding work when it arrives (join the shortest queue, measured in
    work, not in requests); ties go to the lowest rank.  A rank's outstanding
    work drains at `rate` cost units per second (its measured throughput, e.g.
    samples/s).  The routing depends only on the request stream, so every
    rank can compute the same assignment locally with no message on the
    request path; a front end that sees requests one at a time calls `route`
    as they arrive.
    """

    def __init__(self, world: int, homes: Sequence[Sequence[int]], rate: float):
        if world < 1 or not rate > 0:
            raise ValueError("world must be >= 1 and rate > 0")
        for h in homes:
            if not h or any(not 0 <= r < world for r in h):
                raise ValueError(f"bad home ranks {list(h)} for world {world}")
        self.world, self.homes, self.rate = world, [list(h) for h in homes], float(rate)
        self.backlog = [0.0] * world   # outstanding work at time `clock`
        self.clock = 0.0

    def route(self, arrival: float, volume: int, cost: float) -> int:
        if arrival < self.clock:
            raise ValueError("requests must be routed in arrival order")
        drained = (arrival - self.clock) * self.rate
        self.backlog = [max(0.0, b - drained) for b in self.backlog]
        self.clock = arrival
        r = min(self.homes[volume], key=lambda k: (self.backlog[k], k))
        self.backlog[r] += float(cost)
        return r


def request_cost(req) -> float:
    """Estimated work of a serving request: its rays (views x modules x pixels
    come from its matrices and the server's detector), so proportional to the
    sample count for requests of one detector size and similar poses."""
    return float(req.pmats.shape[0] * req.pmats.shape[1])


def route_requests(requests, world: int, homes: Sequence[Sequence[int]], rate: float,
                   cost: Callable = request_cost) -> List[int]:
    """Rank of each request (in the input order), routed in arrival order."""
    router = Router(world, homes, rate)
    order = sorted(range(len(requests)), key=lambda i: (requests[i].arrival, i))
    out = [0] * len(requests)
    for i in order:
        q = requests[i]
        out[i] = router.route(q.arrival, q.volume, cost(q))
    return out


def serve_on_ranks(server, requests, world: int, rank: int, homes: Sequence[Sequence[int]], rate: float,
                   cost: Callable = request_cost, group=None) -> dict:
    """Serve this rank's share of `requests` with `server` (a DRRServer over
    this rank's GPU and the volumes in the same order on every rank), then merge
    the statistics of all ranks: counts and views add up, throughput is over
    the slowest rank's wall time, latency percentiles are over every request."""
    import numpy as np
    import torch.distributed as dist
    ranks = route_requests(requests, world, homes, rate, cost)
    mine = [q for q, r in zip(requests, ranks) if r == rank]
    stats = server.run(mine)
    local = {"completed": stats.completed, "refused": stats.refused, "views": stats.views,
             "wall_s": stats.wall_s, "latencies_ms": list(stats.latencies_ms),
             "served": sorted(q.rid for q in mine if not q.refused)}
    parts = [None] * world
    dist.all_gather_object(parts, local, group=group)
    lat = np.asarray([x for p in parts for x in p["latencies_ms"]]) if any(p["latencies_ms"] for p in parts) \
        else np.zeros(1)
    wall = max(p["wall_s"] for p in parts)
    completed = sum(p["completed"] for p in parts)
    return {
        "requests": len(requests), "completed": completed, "refused": sum(p["refused"] for p in parts),
        "per_rank_requests": [len(p["served"]) for p in parts],
        "served_ids": sorted(i for p in parts for i in p["served"]),
        "throughput_req_s": completed / wall if wall > 0 else 0.0,
        "throughput_views_s": sum(p["views"] for p in parts) / wall if wall > 0 else 0.0,
        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
        "max_ms": float(lat.max()),
    }
