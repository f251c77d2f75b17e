"""View sharding across ranks, run as two gloo processes on the CPU.

Each rank projects its contiguous block of views (with the oracle standing in
for the device, as there is no GPU here), the slices are gathered, and the
result must equal projecting all views in one process.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from ctl_b200.sharding import shard_views


def test_shards_cover_all_views_once():
    for n in (1, 7, 90, 360):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                a, b = shard_views(n, world, r)
                seen.extend(range(a, b))
                assert abs((b - a) - n / world) < 1.0
            assert seen == list(range(n))
    with pytest.raises(ValueError):
        shard_views(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import torch.distributed as dist

    import oracle
    from ctl_b200 import geometry as G
    from ctl_b200 import phantom as Ph
    from ctl_b200.sharding import broadcast_volume, gather_views, project_shard

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # only rank 0 makes the volume; the others receive it
        vol = Ph.ellipsoid_phantom((24, 24, 24), (4, 4, 4), 4, seed=3) if rank == 0 else None
        vol = broadcast_volume(vol, (24, 24, 24)).numpy()
        P = G.circular_flat(7, 750.0, 1000.0, G.FlatDetector(24, 20, 2.0, 2.0))
        _, _, local = project_shard(lambda p: oracle.project_fp64(vol, (4, 4, 4), p, 24, 20, threads=1)[0],
                                    P, world, rank)
        full = gather_views(local, P.shape[0], world, rank)
        if rank == 0:
            q.put(full.numpy())
    finally:
        dist.destroy_process_group()


def _failing_worker(rank, world, port, q):
    """Rank 1 fails after the broadcast, before the view exchange; rank 0 must learn of
    it from the collective (an error, not a hang) and report it."""
    import datetime

    import torch
    import torch.distributed as dist

    from ctl_b200.sharding import broadcast_volume, gather_views

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=10))
    broadcast_volume(np.ones((4, 4, 4), np.float32) if rank == 0 else None, (4, 4, 4))
    if rank == 1:
        os._exit(3)  # the rank dies between steps, with nothing in flight
    try:
        gather_views(torch.zeros((1, 2)), 2, world, rank)
        q.put("no error")
    except Exception as e:  # noqa: BLE001 - any collective error is the detection
        q.put("error: " + type(e).__name__)


def test_two_rank_gather_equals_single_process():
    import oracle
    from ctl_b200 import geometry as G
    from ctl_b200 import phantom as Ph

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    vol = Ph.ellipsoid_phantom((24, 24, 24), (4, 4, 4), 4, seed=3)
    P = G.circular_flat(7, 750.0, 1000.0, G.FlatDetector(24, 20, 2.0, 2.0))
    want, _ = oracle.project_fp64(vol, (4, 4, 4), P, 24, 20, threads=1)
    np.testing.assert_array_equal(got, want)


def test_a_dead_rank_is_reported_by_the_next_collective():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_failing_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    msg = q.get(timeout=120)   # rank 0's verdict arrives well inside the bound: no hang
    for p in procs:
        p.join(timeout=60)
    assert msg.startswith("error"), msg
    assert procs[1].exitcode == 3

