"""Continuous-batching DRR server over resident volumes.

Requests (volume, a few views of arbitrary pose, one detector size) arrive
over time, as in 2D/3D registration and simulation tools that call
RayCasterProjector::project once per pose (examples/regist2d3d/main.cpp,
examples/simTool/mainwindow.cpp:192-217).  Here the volumes stay resident on
the device and requests are batched as they arrive:

* admission: a request is accepted while the device memory of all accepted,
  unfinished requests (their projection matrices and images) stays within the
  budget; otherwise it waits in the arrival queue (or is refused if `refuse`);
* batching: whenever one of `streams` CUDA streams is free, every queued
  request (up to `max_batch`) goes into one batch on it (ctlcu_project_batch:
  one setup launch, then the requests' projection launches), so requests that
  arrive while others run are picked up as soon as a stream frees and their
  work overlaps on the device; the
  batch's matrices go through the stream's pinned staging buffer with a
  non-blocking copy, and its outputs are one allocation sliced per request;
* timing: latency is arrival (host clock) to the end of the request's batch
  on the device (CUDA event), with the device clock tied to the host clock
  at start.

The projections of a request depend only on its own inputs: every ray is
computed independently of the others in its batch, so a result is the same
alone and in any mix (tests/test_gpu_serving.py checks this).
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from .projector import Context, Settings, Volume, torch_stream_handle


# torch's caching allocator serves requests of up to 1 MiB from a separate
# pool of small blocks; one float more than that puts a batch's outputs in the
# large-block pool that DRRServer.reserve() fills
_LARGE_FLOATS = (1 << 20) // 4 + 1


@dataclass
class DRRRequest:
    rid: int
    volume: int             # index into the server's volumes
    pmats: np.ndarray       # (views, modules, 3, 4) float64
    arrival: float          # seconds after the start of the run
    out: object = None      # device tensor (views, modules, rows, channels), set on admission
    done: float = -1.0      # seconds after start when the result was ready on the device
    refused: bool = False

    @property
    def latency(self) -> float:
        return self.done - self.arrival


@dataclass
class ServeStats:
    n: int
    completed: int
    refused: int
    wall_s: float
    views: int
    latencies_ms: List[float] = field(default_factory=list)
    batches: int = 0
    mean_batch: float = 0.0

    def summary(self) -> dict:
        lat = np.asarray(self.latencies_ms) if self.latencies_ms else np.zeros(1)
        return {
            "requests": self.n, "completed": self.completed, "refused": self.refused,
            "throughput_req_s": self.completed / self.wall_s if self.wall_s > 0 else 0.0,
            "throughput_views_s": self.views / self.wall_s if self.wall_s > 0 else 0.0,
            "p50_ms": float(np.percentile(lat, 50)), "p95_ms": float(np.percentile(lat, 95)),
            "p99_ms": float(np.percentile(lat, 99)), "max_ms": float(lat.max()),
            "batches": self.batches, "mean_requests_per_batch": self.mean_batch,
        }


class DRRServer:
    def __init__(self, ctx: Context, volumes: Sequence[Volume], channels: int, rows: int,
                 settings: Optional[Settings] = None, streams: int = 2, max_batch: int = 256,
                 budget_bytes: int = 40 * 10**9, refuse: bool = False, deadline_ms: Optional[float] = None,
                 max_batch_views: Optional[int] = None, reserve_bytes: int = 0):
        import torch
        self.torch = torch
        self.ctx = ctx
        self.volumes = list(volumes)
        self.channels, self.rows = channels, rows
        self.settings = settings or Settings()
        self.streams = [torch.cuda.Stream() for _ in range(streams)]
        self.max_batch = max_batch
        # a batch stops taking requests once it holds this many views (the first request
        # always goes in).  A batch's launches hold the SMs until they are done, so
        # batches on other streams wait behind it; bounding its views bounds that wait.
        self.max_batch_views = max_batch_views
        self.refuse = refuse
        # a queued request that has waited longer than this when a stream frees is
        # refused rather than served late
        self.deadline_s = None if deadline_ms is None else deadline_ms / 1e3
        self.budget_bytes = budget_bytes
        if self._free_budget() <= 0:
            raise ValueError("the resident volumes alone exceed the memory budget")
        # per stream: pinned host staging for a batch's projection matrices and the
        # device buffer they are copied into, grown on demand.  A stream takes its
        # next batch only after the previous one's end event, so a batch never
        # overwrites matrices that are still being copied or read.
        self._pin = [None] * streams
        self._dev = [None] * streams
        if reserve_bytes > 0:
            self.reserve(min(int(reserve_bytes), self._free_budget()))

    def reserve(self, nbytes: int) -> None:
        """Allocate nbytes of device memory for results up front, split over the
        server's streams, and hand it back to torch's caching allocator, which keeps
        it for later allocations on the same stream.  A batch's output allocation is
        then carved from it instead of growing the allocator while requests wait:
        growing it took 20-28 ms per new segment, during which no batch was launched.
        The memory stays reserved for this process (torch.cuda.empty_cache() returns
        whatever is unused)."""
        torch = self.torch
        per = int(nbytes) // len(self.streams)
        if per <= 0:
            return
        for s in self.streams:
            with torch.cuda.stream(s):
                block = torch.empty(per, dtype=torch.uint8, device="cuda")
            del block

    def _free_budget(self) -> int:
        """Budget left for requests after the resident volumes (with their cell arrays)."""
        return self.budget_bytes - sum(v.nbytes for v in self.volumes)

    def _bytes(self, req: DRRRequest) -> int:
        V, M = req.pmats.shape[:2]
        return int(V * M * (self.rows * self.channels * 4 + 96))

    def warm_up(self, typical_pmats: Optional[np.ndarray] = None) -> None:
        """Autotune the sample loop of every volume on a typical request geometry
        (if given), build the arrays it reads and launch once, outside timing."""
        torch = self.torch
        if typical_pmats is not None:
            self.tuned = [self.ctx.autotune(v, typical_pmats, self.channels, self.rows, self.settings)
                          for v in self.volumes]
        P = np.zeros((1, 1, 3, 4))
        P[0, 0, :, :3] = np.eye(3)
        P[0, 0, 2, 3] = 1000.0
        # the device buffers must outlive the asynchronous launches: keep them
        # until the stream is synchronised, and run on torch's current stream
        # so its caching allocator orders any reuse after our kernels
        keep = []
        stream = torch_stream_handle(torch.cuda.current_stream())
        for v in self.volumes:
            out = torch.empty((1, 1, self.rows, self.channels), device="cuda")
            dP = torch.from_numpy(P).cuda()
            keep.append((dP, out))
            self.ctx.project_batch([(v, dP, out)], self.settings, stream=stream)
        # the staging buffers of every stream, before the first request
        for i in range(len(self.streams)):
            self._ensure_stage(i, 1)
        torch.cuda.synchronize()
        self.ctx.sync()

    def _ensure_stage(self, i: int, n: int) -> None:
        """Stream i's staging buffers hold at least n view-modules' matrices."""
        torch = self.torch
        if self._pin[i] is None or self._pin[i].shape[0] < n:
            cap = max(n, 256)
            with torch.cuda.stream(self.streams[i]):
                self._pin[i] = torch.empty((cap, 12), dtype=torch.float64).pin_memory()
                self._dev[i] = torch.empty((cap, 12), dtype=torch.float64, device="cuda")

    def _stage(self, i: int, batch: Sequence[DRRRequest]):
        """The batch's matrices gathered into stream i's pinned staging buffer and
        copied to its device buffer without blocking the host (on the current
        stream, which is stream i): an (n_view_modules, 12) float64 device view."""
        n = sum(int(r.pmats.shape[0] * r.pmats.shape[1]) for r in batch)
        self._ensure_stage(i, n)
        host = self._pin[i].numpy()
        at = 0
        for r in batch:
            k = int(r.pmats.shape[0] * r.pmats.shape[1])
            host[at: at + k] = r.pmats.reshape(k, 12)
            at += k
        dev = self._dev[i][:n]
        dev.copy_(self._pin[i][:n], non_blocking=True)
        return dev

    def run(self, requests: Sequence[DRRRequest]) -> ServeStats:
        """Serve `requests` (arrival times relative to the start) to completion.
        Python's cyclic garbage collector is paused meanwhile: with the previous
        runs' requests and results still alive its full passes took about 100 ms,
        during which no batch was launched and latencies piled up; reference
        counting still frees every request's buffers as before."""
        import gc
        was_enabled = gc.isenabled()
        gc.disable()
        try:
            return self._run(requests)
        finally:
            if was_enabled:
                gc.enable()

    def _run(self, requests: Sequence[DRRRequest]) -> ServeStats:
        torch = self.torch
        reqs = sorted(requests, key=lambda r: r.arrival)
        pending = list(reqs)
        pending.reverse()  # pop() takes the earliest
        queue: List[DRRRequest] = []
        inflight = [None] * len(self.streams)  # (batch, end_event)
        self.budget = self._free_budget()
        used = 0
        done = refused = batches = batched = 0
        torch.cuda.synchronize()
        base = torch.cuda.Event(enable_timing=True)
        base.record(self.streams[0])
        base.synchronize()
        t0 = time.perf_counter()
        while done + refused < len(reqs):
            now = time.perf_counter() - t0
            # arrivals: admit into the queue while the budget allows
            while pending and pending[-1].arrival <= now:
                r = pending[-1]
                need = self._bytes(r)
                if used + need > self.budget:
                    if self.refuse:
                        pending.pop()
                        r.refused = True
                        refused += 1
                        continue
                    break  # wait for memory to free
                pending.pop()
                used += need
                queue.append(r)
            # completions, then new batches on free streams
            for i, s in enumerate(self.streams):
                slot = inflight[i]
                if slot is not None and slot[1].query():
                    ms = base.elapsed_time(slot[1])
                    for r in slot[0]:
                        r.done = ms / 1e3
                        used -= self._bytes(r)
                    done += len(slot[0])
                    inflight[i] = None
                if inflight[i] is None and queue and self.deadline_s is not None:
                    late = time.perf_counter() - t0 - self.deadline_s
                    kept = []
                    for r in queue:
                        if r.arrival < late:
                            r.refused = True
                            refused += 1
                            used -= self._bytes(r)
                        else:
                            kept.append(r)
                    queue = kept
                if inflight[i] is None and queue:
                    take = min(self.max_batch, len(queue))
                    if self.max_batch_views is not None:
                        views, take = 0, 0
                        while take < min(self.max_batch, len(queue)):
                            views += int(queue[take].pmats.shape[0])
                            if take > 0 and views > self.max_batch_views:
                                break
                            take += 1
                    batch, queue = queue[:take], queue[take:]
                    with torch.cuda.stream(s):
                        allP = self._stage(i, batch)
                        # one output allocation per batch; each request keeps its slice.  It
                        # is at least _LARGE_FLOATS long, so that it comes from the caching
                        # allocator's large-block pool, which reserve() fills up front
                        n_vm = allP.shape[0]
                        per = self.rows * self.channels
                        flat = torch.empty(max(n_vm * per, _LARGE_FLOATS), device="cuda")
                        outs = flat[: n_vm * per].view(n_vm, self.rows, self.channels)
                        items, at = [], 0
                        for r in batch:
                            V, M = r.pmats.shape[:2]
                            dP = allP[at: at + V * M].view(V, M, 3, 4)
                            r.out = outs[at: at + V * M].view(V, M, self.rows, self.channels)
                            at += V * M
                            items.append((self.volumes[r.volume], dP, r.out))
                        self.ctx.project_batch(items, self.settings, stream=torch_stream_handle(s))
                        ev = torch.cuda.Event(enable_timing=True)
                        ev.record(s)
                    inflight[i] = (batch, ev)
                    batches += 1
                    batched += len(batch)
        wall = time.perf_counter() - t0
        lat = [1e3 * r.latency for r in reqs if not r.refused]
        views = sum(int(r.pmats.shape[0]) for r in reqs if not r.refused)
        return ServeStats(n=len(reqs), completed=done, refused=refused, wall_s=wall, views=views,
                          latencies_ms=lat, batches=batches, mean_batch=batched / max(batches, 1))


def poisson_requests(rate_hz: float, n: int, n_volumes: int, base_pmats: np.ndarray, seed: int,
                     views=(1, 16), trans_mm: float = 10.0, rot_deg: float = 5.0) -> List[DRRRequest]:
    """Seeded Poisson arrivals; each request asks for 1-16 rigidly perturbed
    copies of the base C-arm view (+-trans_mm, +-rot_deg)."""
    from . import geometry as G
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_hz, n))
    out = []
    for i in range(n):
        nv = int(rng.integers(views[0], views[1] + 1))
        P = G.perturbed_views(base_pmats, nv, rng, trans_mm, rot_deg)
        out.append(DRRRequest(rid=i, volume=int(rng.integers(0, n_volumes)), pmats=P, arrival=float(t[i])))
    return out
