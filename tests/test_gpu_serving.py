"""The continuous-batching DRR server: every request's result is the same
alone and in the mix, and matches the FP64 oracle."""
import numpy as np
import pytest

import oracle
from ctl_b200 import geometry as G
from ctl_b200 import phantom as Ph
from ctl_b200.projector import Context, Settings, VoxelVolume
from ctl_b200.serving import DRRServer, poisson_requests
from tests._common import dequant_bf16, rel_err

pytestmark = pytest.mark.gpu


def _base_view(C=48, R=40):
    det = G.FlatDetector(C, R, 2.4, 2.4)
    return G.circular_flat(1, 750.0, 1200.0, det)[0]  # (modules, 3, 4)


def test_server_results_equal_alone_and_oracle():
    from ctl_b200 import _lib as L
    ctx = Context(0)
    vols = [Ph.ellipsoid_phantom((40, 40, 32), (3, 3, 3), 5, seed=20 + i) for i in range(3)]
    handles = [ctx.volume(VoxelVolume(v, (3, 3, 3)), L.BF16) for v in vols]
    server = DRRServer(ctx, handles, 48, 40, Settings(), streams=2, max_batch=16)
    server.warm_up()
    reqs = poisson_requests(4000.0, 60, len(vols), _base_view(), seed=7, views=(1, 6))
    stats = server.run(reqs)
    assert stats.completed == 60 and stats.refused == 0 and stats.batches >= 2
    assert all(r.done >= r.arrival for r in reqs)
    import torch
    for r in reqs:
        # the same request alone through the same batched path: identical bits
        out = torch.zeros_like(r.out)
        ctx.project_batch([(handles[r.volume], torch.from_numpy(r.pmats).cuda(), out)], Settings())
        ctx.sync()
        np.testing.assert_array_equal(r.out.cpu().numpy(), out.cpu().numpy())
        # and through the single-request kernel
        alone = ctx.project(handles[r.volume], r.pmats, 48, 40, Settings())
        np.testing.assert_allclose(r.out.cpu().numpy(), alone, rtol=1e-6, atol=1e-7)
    for r in reqs[::12]:
        want, _ = oracle.project_fp64(dequant_bf16(vols[r.volume]), (3, 3, 3), r.pmats, 48, 40)
        assert rel_err(r.out.cpu().numpy(), want).max() <= 1e-4
    for h in handles:
        h.release()
    ctx.close()


def test_server_view_cap_bounds_every_batch():
    """With max_batch_views, a batch takes requests until the next would pass the cap (the
    first always goes in); every request is served, with its single-call result."""
    from ctl_b200 import _lib as L
    ctx = Context(0)
    vol = Ph.ellipsoid_phantom((32, 32, 32), (3, 3, 3), 4, seed=9)
    h = ctx.volume(VoxelVolume(vol, (3, 3, 3)), L.BF16)
    server = DRRServer(ctx, [h], 48, 40, Settings(), streams=1, max_batch=64, max_batch_views=7)
    server.warm_up()
    reqs = poisson_requests(1e7, 40, 1, _base_view(), seed=11, views=(1, 9))   # all queued at once
    stats = server.run(reqs)
    assert stats.completed == 40 and stats.refused == 0
    total_views = sum(int(r.pmats.shape[0]) for r in reqs)
    assert stats.batches >= total_views / 9   # no batch beyond 7 views unless one request alone has more
    for r in reqs[::7]:
        alone = ctx.project(h, r.pmats, 48, 40, Settings())
        np.testing.assert_allclose(r.out.cpu().numpy(), alone, rtol=1e-6, atol=1e-7)
    h.release()
    ctx.close()


def test_server_admission_by_budget():
    from ctl_b200 import _lib as L
    ctx = Context(0)
    vol = Ph.ellipsoid_phantom((24, 24, 24), (4, 4, 4), 3, seed=1)
    h = ctx.volume(VoxelVolume(vol, (4, 4, 4)))
    # budget for the volume plus about two requests' images: the rest must wait or be refused
    per_req = 4 * (48 * 40 * 4 + 96)
    server = DRRServer(ctx, [h], 48, 40, Settings(), streams=1, max_batch=8,
                       budget_bytes=h.nbytes + 2 * per_req, refuse=True)
    server.warm_up()
    reqs = poisson_requests(1e6, 20, 1, _base_view(), seed=3, views=(4, 4))
    stats = server.run(reqs)
    assert stats.refused > 0 and stats.completed + stats.refused == 20
    with pytest.raises(ValueError):
        DRRServer(ctx, [h], 48, 40, budget_bytes=1)
    h.release()
    ctx.close()


def test_server_deadline_refuses_late_requests():
    """Far above capacity with a short deadline: requests that waited longer than the
    deadline when a stream freed are refused, and every served request started in time."""
    ctx = Context(0)
    vol = Ph.ellipsoid_phantom((64, 64, 64), (2, 2, 2), 5, seed=2)
    h = ctx.volume(VoxelVolume(vol, (2, 2, 2)))
    server = DRRServer(ctx, [h], 48, 40, Settings(), streams=1, max_batch=2, deadline_ms=2.0)
    server.warm_up()
    reqs = poisson_requests(1e6, 400, 1, _base_view(), seed=5, views=(16, 16))
    stats = server.run(reqs)
    assert stats.refused > 0 and stats.completed > 0 and stats.completed + stats.refused == 400
    served = [r for r in reqs if not r.refused]
    assert all(r.done >= r.arrival for r in served)
    h.release()
    ctx.close()


def test_reserved_server_allocates_nothing_while_serving():
    """With reserve_bytes, the server's result memory is allocated before serving: a run
    grows no device segment (each growth of the caching allocator held up the request
    loop by tens of ms), and its results are the single-call results."""
    import torch

    from ctl_b200 import _lib as L
    ctx = Context(0)
    vol = Ph.ellipsoid_phantom((32, 32, 32), (3, 3, 3), 4, seed=13)
    h = ctx.volume(VoxelVolume(vol, (3, 3, 3)), L.BF16)
    server = DRRServer(ctx, [h], 48, 40, Settings(), streams=2, max_batch=8, reserve_bytes=256 << 20)
    server.warm_up()
    reqs = poisson_requests(20000.0, 50, 1, _base_view(), seed=17, views=(1, 4))
    torch.cuda.synchronize()
    before = torch.cuda.memory_stats().get("segment.all.allocated", 0)
    stats = server.run(reqs)
    after = torch.cuda.memory_stats().get("segment.all.allocated", 0)
    assert stats.completed == 50
    assert after == before, (before, after)
    for r in reqs[::7]:
        alone = ctx.project(h, r.pmats, 48, 40, Settings())
        np.testing.assert_array_equal(r.out.cpu().numpy(), alone)
    del reqs
    h.release()
    ctx.close()
