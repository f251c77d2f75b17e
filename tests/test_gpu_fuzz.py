"""Seeded random cases against the FP64 oracle: geometry, volume and settings
drawn together, every sample loop that serves the case.

Each case draws
  - a volume of 1..40 voxels per axis (some axes 1 voxel thin), voxel sizes
    0.3..2.5 mm per axis, an offset of up to 30% of the extent, values in
    [0, 1) with a zero shell or not;
  - 1..3 views of 1..3 flat modules: a source at 1.5..4 volume radii in a
    random direction, the detector aimed near the volume centre with a random
    roll, 1..40 channels x 1..30 rows whose pitch covers 0.3..1.2 of the
    volume's shadow (so some rays miss), each module shifted and tilted a
    little; the matrix multiplied by a random factor of either sign (the
    projector normalises it, raycasterprojector.cpp:527-541);
  - 1..3 x 1..3 rays per pixel, raySampling 0.1..1.0, volumeUpSampling
    0 (one mean voxel), 1, 2 or 3, trilinear or nearest voxel
    (raycasterprojector.h:27-37);
  - storage F32, BF16 or F16 (16-bit forms are held to the oracle run on the
    stored, de-quantised voxels).

Every case runs the loop CTLCU_KERNEL_AUTO picks and, where they serve it
(trilinear, volumeUpSampling 1), the cell, pair and gather loops by name, all
held to 1e-4 max relative error (denominator max(|oracle|, 1e-3 max|oracle|)).
"""
import math

import numpy as np
import pytest

import oracle
from ctl_b200 import _lib as L
from ctl_b200 import geometry as G
from tests._common import FLOOR, dequant_bf16, dequant_f16

N_CASES = 200
SCALES = (1.0, 3.7, -1.0, -0.25)


def random_case(seed: int) -> dict:
    rng = np.random.default_rng(1000 + seed)
    n = [int(rng.integers(1, 41)) for _ in range(3)]
    if rng.random() < 0.2:
        n[int(rng.integers(0, 3))] = 1
    voxel = tuple(float(v) for v in rng.uniform(0.3, 2.5, 3))
    extent = np.array(n) * np.array(voxel)
    offset = tuple(float(o) for o in rng.uniform(-0.3, 0.3, 3) * extent)
    vol = rng.random((n[2], n[1], n[0]), dtype=np.float32)
    if rng.random() < 0.5 and min(n) > 2:
        vol[0], vol[-1], vol[:, 0], vol[:, -1], vol[:, :, 0], vol[:, :, -1] = 0, 0, 0, 0, 0, 0
    radius = 0.5 * float(np.linalg.norm(extent))
    centre = np.array(offset)
    V, M = int(rng.integers(1, 4)), int(rng.integers(1, 4))
    channels, rows = int(rng.integers(1, 41)), int(rng.integers(1, 31))
    P = np.empty((V, M, 3, 4))
    for v in range(V):
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        sid = radius * rng.uniform(1.5, 4.0)
        src = centre + sid * d
        sdd = sid * rng.uniform(1.2, 2.5)
        aim = centre + rng.uniform(-0.2, 0.2, 3) * radius
        principal = aim - src
        up = rng.normal(size=3)
        if abs(np.dot(up, principal)) > 0.95 * np.linalg.norm(up) * np.linalg.norm(principal):
            up = np.cross(principal, [1.0, 0.0, 0.0]) + np.cross(principal, [0.0, 1.0, 0.0])
        # the volume's shadow is about 2 radius * sdd / sid wide on the detector
        cover = rng.uniform(0.3, 1.2)
        pitch_x = 2 * radius * sdd / sid * cover / channels
        pitch_y = 2 * radius * sdd / sid * cover / rows * rng.uniform(0.5, 2.0)
        for m in range(M):
            R = G.camera_rotation(principal, up)
            if M > 1:
                R = G.rot_axis(np.array([0.0, 1.0, 0.0]), math.radians(8.0 * (m - (M - 1) / 2))) @ R
            cx = (channels - 1) / 2.0 + (m - (M - 1) / 2) * channels * 0.5 + rng.uniform(-1, 1)
            cy = (rows - 1) / 2.0 + rng.uniform(-1, 1)
            K = G.intrinsic(sdd, pitch_x, pitch_y, cx, cy)
            P[v, m] = G.normalized(G.compose(K, R, src)) * SCALES[int(rng.integers(0, len(SCALES)))]
    interpolate = bool(rng.random() < 0.8)
    ups = int(rng.choice([0, 1, 1, 1, 2, 3]))
    case = dict(seed=seed, volume=vol, voxel=voxel, offset=offset, pmats=P, channels=channels, rows=rows,
                rays=(int(rng.integers(1, 4)), int(rng.integers(1, 4))),
                ray_sampling=float(rng.uniform(0.1, 1.0)), upsampling=ups, interpolate=interpolate,
                storage=[L.F32, L.F32, L.BF16, L.F16][int(rng.integers(0, 4))])
    return case


def _stored(case):
    vol = case["volume"]
    if case["storage"] == L.BF16:
        return dequant_bf16(vol)
    if case["storage"] == L.F16:
        return dequant_f16(vol)
    return vol


def _oracle(case):
    want, _ = oracle.project_fp64(_stored(case), case["voxel"], case["pmats"], case["channels"], case["rows"],
                                  offset_mm=case["offset"], rays=case["rays"], ray_sampling=case["ray_sampling"],
                                  upsampling=case["upsampling"], interpolate=case["interpolate"])
    return want


def _max_rel(got, want):
    want = np.asarray(want, np.float64)
    d = np.maximum(np.abs(want), FLOOR * np.abs(want).max()) if np.abs(want).max() > 0 else 1.0
    return float((np.abs(np.asarray(got, np.float64) - want) / d).max())


def test_random_cases_are_valid_inputs():
    """The generator: finite matrices with a non-singular M, and an oracle result
    that sees the volume in most cases (CPU only)."""
    hits = 0
    for seed in range(N_CASES):
        c = random_case(seed)
        assert np.isfinite(c["pmats"]).all()
        for P in c["pmats"].reshape(-1, 3, 4):
            assert abs(np.linalg.det(P[:, :3])) > 1e-12
        hits += bool(np.abs(_oracle(c)).max() > 0)
    assert hits >= 0.8 * N_CASES


@pytest.fixture(scope="module")
def ctx():
    from ctl_b200.projector import Context
    c = Context(0)
    yield c
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(N_CASES))
def test_random_case_matches_oracle(ctx, seed):
    from ctl_b200.projector import Settings, VoxelVolume
    c = random_case(seed)
    want = _oracle(c)
    h = ctx.volume(VoxelVolume(c["volume"], c["voxel"], c["offset"]), c["storage"])
    loops = [L.KERNEL_AUTO]
    if c["interpolate"] and c["upsampling"] == 1:
        loops += [L.KERNEL_CELLS, L.KERNEL_PAIRS, L.KERNEL_GATHER]
    for k in loops:
        s = Settings(rays_per_pixel=list(c["rays"]), ray_sampling=c["ray_sampling"],
                     volume_upsampling=c["upsampling"], interpolate=c["interpolate"], kernel=k)
        got = ctx.project(h, c["pmats"], c["channels"], c["rows"], s)
        err = _max_rel(got, want)
        assert err <= 1e-4, (seed, k, err, {x: c[x] for x in c if x not in ("volume", "pmats")})
    h.release()


def _batchable(seed: int) -> bool:
    c = random_case(seed)
    return c["interpolate"] and c["upsampling"] == 1


@pytest.mark.gpu
@pytest.mark.parametrize("batch", range(6))
def test_random_batch_equals_single_calls(ctx, batch):
    """Eight random cases (different volumes, storage types, detectors, modules and
    view counts) in one batch, one settings for all: ctlcu_project_batch and a plan
    in each form give every request the bits of its single call."""
    import torch
    from ctl_b200.projector import Settings, VoxelVolume
    rng = np.random.default_rng(77 + batch)
    seeds = [s for s in range(N_CASES) if _batchable(s)]
    pick = [seeds[int(i)] for i in rng.choice(len(seeds), 8, replace=False)]
    kernel = [L.KERNEL_CELLS, L.KERNEL_PAIRS][batch % 2]
    s = Settings(rays_per_pixel=[int(rng.integers(1, 3)), int(rng.integers(1, 3))],
                 ray_sampling=float(rng.uniform(0.15, 0.8)), kernel=kernel)
    reqs, singles, handles = [], [], []
    for seed in pick:
        c = random_case(seed)
        h = ctx.volume(VoxelVolume(c["volume"], c["voxel"], c["offset"]), c["storage"])
        handles.append(h)
        V, M = c["pmats"].shape[:2]
        out = torch.full((V, M, c["rows"], c["channels"]), float("nan"), device="cuda")
        reqs.append((h, torch.from_numpy(c["pmats"]).cuda(), out))
        singles.append(ctx.project(h, c["pmats"], c["channels"], c["rows"], s))
    ctx.project_batch(reqs, s)
    ctx.sync()
    for (_, _, out), want in zip(reqs, singles):
        np.testing.assert_array_equal(out.cpu().numpy(), want)
    for form in (L.PLAN_PERSISTENT, L.PLAN_GRIDS):
        for _, _, out in reqs:
            out.fill_(float("nan"))
        plan = ctx.plan(reqs, s, form=form)
        plan.launch()
        ctx.sync()
        for (_, _, out), want in zip(reqs, singles):
            np.testing.assert_array_equal(out.cpu().numpy(), want)
        plan.close()
    del reqs
    for h in handles:
        h.release()
