"""The multi-GPU helpers of ctl_b200.sharding on a real GPU data path: NCCL,
device tensors and the C ABI together.

Every GPU call available here has one GPU, so the process group has one rank;
the collectives then move data on the device through NCCL exactly as they do
with more ranks, without any exchange between GPUs.  The test runs in a child
process so that its process group cannot outlive it.  It checks that
broadcast_volume -> ctlcu_volume_create from device memory -> project_shard ->
gather_views gives the bits of a plain single-process projection, and that
serve_on_ranks serves every request once with single-call results."""
import os
import socket
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import datetime, sys
import numpy as np, torch, torch.distributed as dist
sys.path.insert(0, sys.argv[1])
from ctl_b200 import _lib as L
from ctl_b200 import geometry as G, workloads as W
from ctl_b200.projector import Context, Settings, VoxelVolume
from ctl_b200.serving import DRRServer, poisson_requests
from ctl_b200.sharding import broadcast_volume, gather_views, project_shard, serve_on_ranks, volume_homes

torch.cuda.set_device(0)
dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=60), device_id=torch.device("cuda", 0))
rank, world = dist.get_rank(), dist.get_world_size()
job = W.c1()
vol = broadcast_volume(job.volume if rank == 0 else None, job.volume.shape, device="cuda:0")
assert vol.is_cuda and torch.equal(vol.cpu(), torch.from_numpy(job.volume))
ctx = Context(0)
h = ctx.volume(VoxelVolume(vol, job.voxel))
start, stop, mine = project_shard(lambda P: ctx.project(h, torch.from_numpy(P).cuda(), job.channels, job.rows,
                                                        Settings()), job.pmats, world, rank)
full = gather_views(mine, job.pmats.shape[0], world, rank)
want = ctx.project_volume(VoxelVolume(job.volume, job.voxel), job.pmats, job.channels, job.rows, Settings())
assert full.shape[0] == job.pmats.shape[0]
np.testing.assert_array_equal(full.cpu().numpy(), want)
# serving on the ranks: every request served exactly once, with its single-call result
det = G.FlatDetector(48, 40, 2.4, 2.4)
base = G.circular_flat(1, 750.0, 1200.0, det)[0]
small = ctx.volume(VoxelVolume(W.c1().volume, (2.0, 2.0, 2.0)))
server = DRRServer(ctx, [small], 48, 40, Settings(), streams=2, max_batch=8)
server.warm_up()
reqs = poisson_requests(5000.0, 30, 1, base, seed=3, views=(1, 4))
summary = serve_on_ranks(server, reqs, world, rank, volume_homes(1, world), rate=1e5)
assert summary["served_ids"] == list(range(30)) and summary["completed"] == 30, summary
for r in reqs[::5]:
    np.testing.assert_array_equal(r.out.cpu().numpy(), ctx.project(small, r.pmats, 48, 40, Settings()))
del reqs
h.release(); small.release(); ctx.close()
dist.destroy_process_group()
print("NCCL-PATH-OK")
'''


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharding_helpers_over_nccl_on_the_device():
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()), RANK="0", WORLD_SIZE="1",
               LOCAL_RANK="0")
    r = subprocess.run([sys.executable, "-c", CHILD, ROOT], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "NCCL-PATH-OK" in r.stdout, (r.returncode, r.stdout[-2000:], r.stderr[-4000:])
