"""Batches and serving across ranks (host logic; two gloo processes on the CPU).

Longest-first assignment of uneven requests, routing of serving requests to
the least-loaded rank that holds the volume, and the merge of per-rank
serving statistics.  In the two-process test a stand-in server projects with
the FP64 oracle in place of the device.
"""
import itertools
import os
import socket
import time

import numpy as np
import pytest
import torch.multiprocessing as mp

from ctl_b200.sharding import Router, lpt_assign, route_requests, shard_batch, volume_homes


def _best_makespan(costs, world):
    best = float("inf")
    for assign in itertools.product(range(world), repeat=len(costs)):
        load = [0.0] * world
        for c, r in zip(costs, assign):
            load[r] += c
        best = min(best, max(load))
    return best


def test_lpt_is_within_grahams_bound():
    rng = np.random.default_rng(0)
    for trial in range(60):
        world = int(rng.integers(2, 4))
        n = int(rng.integers(1, 9))
        costs = [float(x) for x in rng.integers(1, 100, n)]
        ranks = lpt_assign(costs, world)
        assert len(ranks) == n and all(0 <= r < world for r in ranks)
        load = [sum(c for c, r in zip(costs, ranks) if r == k) for k in range(world)]
        assert max(load) <= (4.0 / 3.0 - 1.0 / (3 * world)) * _best_makespan(costs, world) + 1e-9
        assert lpt_assign(costs, world) == ranks  # deterministic


def test_shard_batch_partitions_the_requests():
    costs = [5, 1, 9, 9, 2, 7, 3]
    parts = [shard_batch(costs, 3, r) for r in range(3)]
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    assert all(p == sorted(p) for p in parts)
    with pytest.raises(ValueError):
        shard_batch(costs, 3, 3)
    assert lpt_assign([], 2) == []


def test_volume_homes():
    assert volume_homes(3, 2) == [[0, 1], [0, 1], [0, 1]]
    assert volume_homes(4, 3, replicas=1) == [[0], [1], [2], [0]]
    assert volume_homes(2, 4, replicas=2) == [[0, 1], [1, 2]]


class _Req:
    def __init__(self, rid, volume, arrival, views=4):
        self.rid, self.volume, self.arrival = rid, volume, arrival
        self.pmats = np.zeros((views, 1, 3, 4))


def test_router_respects_homes_and_balances_work():
    # volumes on one rank each: every request goes home
    reqs = [_Req(i, i % 4, 0.001 * i) for i in range(40)]
    ranks = route_requests(reqs, 2, volume_homes(4, 2, replicas=1), rate=1e3)
    assert all(r == q.volume % 2 for q, r in zip(reqs, ranks))
    # replicated volumes, a burst: equal requests alternate between the ranks
    burst = [_Req(i, 0, 0.0) for i in range(10)]
    ranks = route_requests(burst, 2, volume_homes(1, 2), rate=1.0)
    assert ranks == [0, 1] * 5
    # replicated, arrivals far apart: the work drains in between, all go to rank 0
    sparse = [_Req(i, 0, float(i)) for i in range(10)]
    assert route_requests(sparse, 2, volume_homes(1, 2), rate=1e6) == [0] * 10
    # a big request fills rank 0, so the small ones after it go to rank 1
    mixed = [_Req(0, 0, 0.0, views=64)] + [_Req(i, 0, 0.0, views=1) for i in range(1, 5)]
    assert route_requests(mixed, 2, volume_homes(1, 2), rate=1.0) == [0, 1, 1, 1, 1]
    with pytest.raises(ValueError):
        Router(2, [[2]], 1.0)
    r = Router(2, [[0, 1]], 1.0)
    r.route(1.0, 0, 1.0)
    with pytest.raises(ValueError):
        r.route(0.5, 0, 1.0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


VOX = (4.0, 4.0, 4.0)


def _volumes():
    from ctl_b200 import phantom as Ph
    return [Ph.ellipsoid_phantom((16, 16, 16), VOX, 3, seed=30 + v) for v in range(3)]


def _requests():
    from ctl_b200 import geometry as G
    from ctl_b200.serving import DRRRequest
    base = G.circular_flat(1, 500.0, 800.0, G.FlatDetector(12, 10, 3.0, 3.0))[0]
    rng = np.random.default_rng(9)
    out, t = [], 0.0
    for i in range(14):
        t += float(rng.exponential(0.002))
        P = G.perturbed_views(base, int(rng.integers(1, 4)), rng, 5.0, 3.0)
        out.append(DRRRequest(rid=i, volume=int(rng.integers(0, 3)), pmats=P, arrival=t))
    return out


class _OracleServer:
    """Stand-in for a DRRServer on a GPU: serves its requests in arrival order
    with the FP64 oracle and records the results."""

    def __init__(self, volumes):
        self.volumes = volumes
        self.results = {}

    def run(self, requests):
        import oracle
        from ctl_b200.serving import ServeStats
        t0 = time.perf_counter()
        lat = []
        for q in sorted(requests, key=lambda q: q.arrival):
            self.results[q.rid], _ = oracle.project_fp64(self.volumes[q.volume], VOX, q.pmats, 12, 10, threads=1)
            q.done = q.arrival + 1e-3
            lat.append(1e3 * q.latency)
        return ServeStats(n=len(requests), completed=len(requests), refused=0, wall_s=time.perf_counter() - t0,
                          views=sum(int(q.pmats.shape[0]) for q in requests), latencies_ms=lat)


def _serving_worker(rank, world, port, q):
    import torch.distributed as dist

    from ctl_b200.sharding import serve_on_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        server = _OracleServer(_volumes())
        reqs = _requests()
        summary = serve_on_ranks(server, reqs, world, rank, volume_homes(3, world), rate=2000.0)
        parts = [None] * world
        dist.all_gather_object(parts, server.results)
        if rank == 0:
            merged = {}
            for p in parts:
                assert not set(p) & set(merged), "a request was served twice"
                merged.update(p)
            q.put((summary, merged))
    finally:
        dist.destroy_process_group()


def test_two_rank_serving_serves_every_request_once_with_oracle_results():
    import oracle
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_serving_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    summary, results = q.get(timeout=180)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    reqs = _requests()
    assert summary["requests"] == len(reqs) == summary["completed"]
    assert summary["served_ids"] == list(range(len(reqs)))
    assert sum(summary["per_rank_requests"]) == len(reqs) and min(summary["per_rank_requests"]) > 0
    assert summary["p99_ms"] == pytest.approx(1.0)
    vols = _volumes()
    for r in reqs:
        want, _ = oracle.project_fp64(vols[r.volume], VOX, r.pmats, 12, 10, threads=1)
        np.testing.assert_array_equal(results[r.rid], want)
