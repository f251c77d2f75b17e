"""Max and mean relative error per benchmark configuration, against the FP64
oracle and against the reference's own ray caster on identical inputs.

The reference's kernel is raycasterprojector_interp.cl:18-72 compiled for the
CPU (oracle/_ref): FP32 sample positions from the source, the OpenCL linear
filter, an FP64 sum.  Its own distance from the FP64 oracle is printed beside
ours.  Cases, at sizes the CPU checkers finish in seconds:

  C1  64^3 -> 90 x 128^2: all 90 views, F32 and BF16 storage
  C2  256^3 -> 512^2: 16 evenly spaced views of 360, F32 / BF16 / F16 storage
  C3  512^3 -> 64 x 16^2 helical: the first and last view of each of the 4
      turns, and at the same views every precision form -- the software FP32
      trilinear cell loop with Kahan, FP64 and plain FP32 accumulation, the
      gather loop, the hardware texture filter, BF16 and F16 storage
  C4  one view of every one of the 64 uneven volumes, F32 and BF16, all in one
      batch
  C5  two perturbed views of 256^2 on each of the 8 resident BF16 volumes, one
      batch

Bars (every form held to its own): 1e-4 max against the FP64 oracle for the
software loops with Kahan or FP64 accumulation; 2e-3 for plain FP32
accumulation; 2e-2 max and 2e-3 mean for the texture filter (8-bit fractional
weights).  16-bit storage is compared with the oracle run on the stored
(de-quantised) volume; its quantisation error against the FP32 volume is
printed beside it.  Against the reference kernel the difference must stay
within the reference's own error envelope (its distance from the oracle plus
our bar), and the reference's distance from the oracle must stay within 1e-3
(the FP32-vs-FP64 gap of its sample positions), which pins the oracle to the
reference at full size.  `pytest -s` shows one PARITY line per case."""
import numpy as np
import pytest
import torch

import oracle
from ctl_b200 import _lib as L
from ctl_b200 import geometry as G
from ctl_b200 import workloads as W
from ctl_b200.projector import Context, Settings, VoxelVolume
from tests._common import FLOOR, dequant_bf16, dequant_f16

pytestmark = pytest.mark.gpu

STORAGE = {L.F32: "f32", L.BF16: "bf16", L.F16: "f16"}


def _stored(vol, storage):
    if storage == L.BF16:
        return dequant_bf16(vol)
    if storage == L.F16:
        return dequant_f16(vol)
    return vol


def _errs(a, b, d):
    e = np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)) / d
    return float(e.max()), float(e.mean())


def _check(name, got, want, ref=None, bar=1e-4, mean_bar=None, extra=""):
    """got vs the FP64 oracle `want` (and the reference kernel `ref` when given),
    all measured with the oracle's denominator max(|want|, 1e-3 max|want|)."""
    want = np.asarray(want, np.float64)
    d = np.maximum(np.abs(want), FLOOR * np.abs(want).max())
    mx, mn = _errs(got, want, d)
    line = f"\nPARITY {name}: vs FP64 oracle max {mx:.2e} mean {mn:.2e}"
    if ref is not None:
        rmx, rmn = _errs(got, ref, d)
        omx, omn = _errs(ref, want, d)
        line += f" | vs reference kernel max {rmx:.2e} mean {rmn:.2e} | reference vs oracle max {omx:.2e} mean {omn:.2e}"
    print(line + f" ({want.size} pixels){extra}")
    assert mx <= bar, (name, mx)
    if mean_bar is not None:
        assert mn <= mean_bar, (name, mn)
    if ref is not None:
        assert rmx <= omx + bar, (name, rmx, omx)
        # the oracle pinned to the reference kernel at full size: they differ only by
        # the reference's FP32 sample positions and filter arithmetic
        assert omx <= 1e-3, (name, omx)


def _ref(*args, **kw):
    return oracle.project_ref(*args, **kw) if oracle.ref_available() else None


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
    vol = _stored(job.volume, storage)
    want, _ = oracle.project_fp64(vol, job.voxel, job.pmats, job.channels, job.rows)
    ref = _ref(vol, job.voxel, job.pmats, job.channels, job.rows)
    _check(f"C1 64^3 -> 90 x 128^2, {STORAGE[storage]} storage, all 90 views", got, want, ref)
    h.release()


@pytest.mark.parametrize("storage", [L.F32, L.BF16, L.F16])
def test_c2_spread_views(ctx, storage):
    job = W.c2()
    views = np.linspace(0, 359, 16).round().astype(int)
    P = np.ascontiguousarray(job.pmats[views])
    h = ctx.volume(VoxelVolume(job.volume, job.voxel), storage)
    got = ctx.project(h, P, job.channels, job.rows, Settings())
    vol = _stored(job.volume, storage)
    want, _ = oracle.project_fp64(vol, job.voxel, P, job.channels, job.rows)
    ref = _ref(vol, job.voxel, P, job.channels, job.rows)
    extra = ""
    if storage != L.F32:
        w32, _ = oracle.project_fp64(job.volume, job.voxel, P, job.channels, job.rows)
        d = np.maximum(np.abs(w32), FLOOR * np.abs(w32).max())
        qmx, qmn = _errs(want, w32, d)
        extra = f"; quantisation of the volume itself: max {qmx:.2e} mean {qmn:.2e}"
    _check(f"C2 256^3 -> 512^2, {STORAGE[storage]} storage, 16 of 360 views", got, want, ref, extra=extra)
    h.release()


# the first and last view of each of the 4 turns of 360 views
C3_VIEWS = [0, 359, 360, 719, 720, 1079, 1080, 1439]

C3_FORMS = [
    # (name, settings, storage, max bar, mean bar)
    ("cells, Kahan accumulator (default)", dict(), L.F32, 1e-4, None),
    ("cells, FP64 accumulator", dict(accum=L.ACCUM_FP64), L.F32, 1e-4, None),
    ("cells, plain FP32 accumulator", dict(accum=L.ACCUM_FP32), L.F32, 2e-3, None),
    ("gather (8 scalar loads), Kahan", dict(kernel=L.KERNEL_GATHER), L.F32, 1e-4, None),
    ("hardware texture filter, FP64 accumulator", dict(interp_mode=L.INTERP_TEXTURE, accum=L.ACCUM_FP64), L.F32,
     2e-2, 2e-3),
    ("cells, Kahan, BF16 storage", dict(), L.BF16, 1e-4, None),
    ("cells, Kahan, F16 storage", dict(), L.F16, 1e-4, None),
]


@pytest.fixture(scope="module")
def c3_case():
    job = W.c3(device="cuda")
    vol = job.volume.cpu().numpy()
    P = np.ascontiguousarray(job.pmats[C3_VIEWS])
    want = {}
    ref = {}
    for storage in (L.F32, L.BF16, L.F16):
        v = _stored(vol, storage)
        want[storage], _ = oracle.project_fp64(v, job.voxel, P, job.channels, job.rows)
        ref[storage] = _ref(v, job.voxel, P, job.channels, job.rows)
    yield job, vol, P, want, ref
    del job
    torch.cuda.empty_cache()


@pytest.mark.parametrize("form", C3_FORMS, ids=[f[0] for f in C3_FORMS])
def test_c3_precision_forms(ctx, c3_case, form):
    name, kw, storage, bar, mean_bar = form
    job, vol, P, want, ref = c3_case
    h = ctx.volume(VoxelVolume(job.volume, job.voxel), storage)
    got = ctx.project(h, P, job.channels, job.rows, Settings(**kw))
    extra = ""
    if storage != L.F32:
        d = np.maximum(np.abs(want[L.F32]), FLOOR * np.abs(want[L.F32]).max())
        qmx, qmn = _errs(want[storage], want[L.F32], d)
        extra = f"; quantisation of the volume itself: max {qmx:.2e} mean {qmn:.2e}"
    _check(f"C3 512^3 -> 64 x 16^2 helical, {STORAGE[storage]} storage, {name}, first and last view of each "
           f"turn", got, want[storage], ref[storage], bar=bar, mean_bar=mean_bar, extra=extra)
    h.release()
    torch.cuda.empty_cache()


@pytest.mark.parametrize("storage", [L.F32, L.BF16])
def test_c4_every_volume_in_one_batch(ctx, storage):
    jobs = W.c4()
    reqs, keep = [], []
    for j in jobs:
        P = np.ascontiguousarray(j.pmats[[j.pmats.shape[0] // 2]])
        h = ctx.volume(VoxelVolume(j.volume, j.voxel), storage)
        out = torch.empty((1, 1, j.rows, j.channels), device="cuda")
        reqs.append((h, torch.from_numpy(P).cuda(), out))
        keep.append((j, P, h, out))
    ctx.project_batch(reqs, Settings())
    ctx.sync()
    gots, wants, refs = [], [], []
    for j, P, h, out in keep:
        vol = _stored(j.volume.cpu().numpy(), storage)
        want, _ = oracle.project_fp64(vol, j.voxel, P, j.channels, j.rows)
        ref = _ref(vol, j.voxel, P, j.channels, j.rows)
        got = out.cpu().numpy()
        # each volume against its own oracle scale, then all 64 together
        d = np.maximum(np.abs(want), FLOOR * np.abs(want).max())
        gots.append((got / d).ravel())
        wants.append((want / d).ravel())
        refs.append(None if ref is None else (ref / d).ravel())
        h.release()
    got, want = np.concatenate(gots), np.concatenate(wants)
    ref = None if refs[0] is None else np.concatenate(refs)
    # already normalised: the denominator is 1 wherever the oracle is below its floor
    mx, mn = _errs(got, want, 1.0)
    line = f"\nPARITY C4 64 uneven volumes, {STORAGE[storage]} storage, one view of each, one batch: " \
           f"vs FP64 oracle max {mx:.2e} mean {mn:.2e}"
    if ref is not None:
        rmx, rmn = _errs(got, ref, 1.0)
        omx, omn = _errs(ref, want, 1.0)
        line += f" | vs reference kernel max {rmx:.2e} mean {rmn:.2e} | reference vs oracle max {omx:.2e} " \
                f"mean {omn:.2e}"
        assert rmx <= omx + 1e-4
        assert omx <= 1e-3
    print(line + f" ({got.size} pixels)")
    assert mx <= 1e-4
    del reqs, keep
    torch.cuda.empty_cache()


def test_c5_requests_on_every_bf16_volume(ctx):
    vols = W.c5_volumes()
    base = W.c5_base_view()
    rng = np.random.default_rng(55)
    reqs, keep = [], []
    for i, v in enumerate(vols):
        P = G.perturbed_views(base, 2, rng, 10.0, 5.0)
        h = ctx.volume(VoxelVolume(v, (1.0, 1.0, 1.0)), L.BF16)
        out = torch.empty((2, 1, 256, 256), device="cuda")
        reqs.append((h, torch.from_numpy(P).cuda(), out))
        keep.append((v, P, h, out))
    ctx.project_batch(reqs, Settings())
    ctx.sync()
    for i, (v, P, h, out) in enumerate(keep):
        vol = dequant_bf16(v.cpu().numpy())
        want, _ = oracle.project_fp64(vol, (1.0, 1.0, 1.0), P, 256, 256)
        ref = _ref(vol, (1.0, 1.0, 1.0), P, 256, 256)
        _check(f"C5 request on 256^3 bf16 volume {i} (2 perturbed views of 256^2, one batch of 8)",
               out.cpu().numpy(), want, ref)
        h.release()
