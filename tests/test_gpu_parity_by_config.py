"""Max and mean relative error against the FP64 oracle for each benchmark configuration,
at sizes the oracle finishes in seconds: all of C1, evenly spaced full-size views of C2
and C3, the first C4 volumes through one batch, and C5 requests on BF16 volumes.  Each
result is printed (pytest -s shows the lines) and held to the 1e-4 bar; 16-bit storage
is compared with the oracle on the stored (de-quantised) volume."""
import numpy as np
import pytest
import torch

import oracle
from ctl_b200 import _lib as L
from ctl_b200 import geometry as G
from ctl_b200 import workloads as W
from ctl_b200.projector import Context, Settings, VoxelVolume
from tests._common import dequant_bf16, rel_err

pytestmark = pytest.mark.gpu

STORAGE = {L.F32: "f32", L.BF16: "bf16", L.F16: "f16"}


def _stored(vol, storage):
    if storage == L.BF16:
        return dequant_bf16(vol)
    if storage == L.F16:
        return vol.astype(np.float16).astype(np.float32)
    return vol


def _check(name, got, want):
    e = rel_err(got, want)
    print(f"\nPARITY {name}: max {e.max():.2e}  mean {e.mean():.2e}  ({e.size} pixels)")
    assert e.max() <= 1e-4, name


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("storage", [L.F32, L.BF16])
def test_c1_every_view(ctx, storage):
    job = W.c1()
    h = ctx.volume(VoxelVolume(job.volume, job.voxel), storage)
    got = ctx.project(h, job.pmats, job.channels, job.rows, Settings())
    want, _ = oracle.project_fp64(_stored(job.volume, storage), job.voxel, job.pmats, job.channels, job.rows)
    _check(f"C1 64^3 -> 90 x 128^2, {STORAGE[storage]} storage, all 90 views", got, want)
    h.release()


@pytest.mark.parametrize("storage", [L.F32, L.BF16, L.F16])
def test_c2_spread_views(ctx, storage):
    job = W.c2()
    P = np.ascontiguousarray(job.pmats[[0, 120, 240, 359]])
    h = ctx.volume(VoxelVolume(job.volume, job.voxel), storage)
    got = ctx.project(h, P, job.channels, job.rows, Settings())
    want, _ = oracle.project_fp64(_stored(job.volume, storage), job.voxel, P, job.channels, job.rows)
    _check(f"C2 256^3 -> 512^2, {STORAGE[storage]} storage, views 0/120/240/359 of 360", got, want)
    h.release()


def test_c3_helical_views(ctx):
    job = W.c3(device="cuda")
    vol = job.volume.cpu().numpy()
    P = np.ascontiguousarray(job.pmats[[0, 480, 960, 1439]])
    h = ctx.volume(VoxelVolume(job.volume, job.voxel))
    got = ctx.project(h, P, job.channels, job.rows, Settings())
    want, _ = oracle.project_fp64(vol, job.voxel, P, job.channels, job.rows)
    _check("C3 512^3 -> 64 x 16^2 helical, f32 storage, views 0/480/960/1439 of 1440", got, want)
    h.release()
    del job
    torch.cuda.empty_cache()


def test_c4_uneven_volumes_in_one_batch(ctx):
    jobs = W.c4(n_volumes=3)
    reqs, keep = [], []
    for j in jobs:
        P = np.ascontiguousarray(j.pmats[[0, j.pmats.shape[0] // 2]])
        h = ctx.volume(VoxelVolume(j.volume, j.voxel))
        out = torch.empty((2, 1, j.rows, j.channels), device="cuda")
        reqs.append((h, torch.from_numpy(P).cuda(), out))
        keep.append((j, P, h, out))
    ctx.project_batch(reqs, Settings())
    ctx.sync()
    for j, P, h, out in keep:
        want, _ = oracle.project_fp64(j.volume.cpu().numpy(), j.voxel, P, j.channels, j.rows)
        _check(f"C4 {j.name} (2 views, one batch with the others)", out.cpu().numpy(), want)
        h.release()


def test_c5_requests_on_bf16_volumes(ctx):
    vols = W.c5_volumes(n=2)
    base = W.c5_base_view()
    rng = np.random.default_rng(55)
    reqs, keep = [], []
    for i, v in enumerate(vols):
        P = G.perturbed_views(base, 3, rng, 10.0, 5.0)
        h = ctx.volume(VoxelVolume(v, (1.0, 1.0, 1.0)), L.BF16)
        out = torch.empty((3, 1, 256, 256), device="cuda")
        reqs.append((h, torch.from_numpy(P).cuda(), out))
        keep.append((v, P, h, out))
    ctx.project_batch(reqs, Settings())
    ctx.sync()
    for i, (v, P, h, out) in enumerate(keep):
        want, _ = oracle.project_fp64(dequant_bf16(v.cpu().numpy()), (1.0, 1.0, 1.0), P, 256, 256)
        _check(f"C5 request on 256^3 bf16 volume {i} (3 perturbed views of 256^2, one batch)",
               out.cpu().numpy(), want)
        h.release()
