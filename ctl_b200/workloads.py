"""The benchmark configurations as seeded synthetic workloads.

  c1  64^3 f32 (2 mm), 10 ellipsoids; circular, 90 views over 360 deg,
      SID 750, SDD 1000, 128 x 128 flat detector at 1.0 mm
  c2  256^3 f32 (1 mm), 40 ellipsoids; short scan 200 deg + fan, 360 views,
      512 x 512 at 0.6 mm, SID 750, SDD 1200, seeded +-0.5 mm / +-0.2 deg jitter
  c3  512^3 (0.5 mm), ellipsoids + 1% Gaussian texture; helical, 1440 views over
      4 turns, SID 570, SDD 1040, curved detector of 64 flat modules of
      16 channels x 16 rows at 1.0 mm (1024 x 16); the 4 turns span the
      volume's z extent (the table feed is otherwise unspecified)
  c4  64 volumes, edges drawn from {96, 128, ..., 256} per axis, f32 or BF16,
      30-360 views each of circular cone beam (SID 750, SDD 1000), detectors
      from 256 x 256 to 768 x 512 at 0.5-1.0 mm
  c5  8 resident 256^3 BF16 volumes; requests of 1-16 views of a 256 x 256
      detector at 1.2 mm, posed as the c2 base view with a +-10 mm / +-5 deg
      rigid perturbation, Poisson arrivals at 2000/s

No public dataset is involved; seeds are fixed here.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List

import numpy as np

from . import geometry as G
from . import phantom as Ph


def phantom_device(shape_xyz, voxel_mm, n_ellipsoids: int, seed: int, texture: float = 0.0,
                   device: str = "cuda"):
    """ellipsoid_phantom() evaluated with torch on `device` (same seeded
    parameters; float32 arithmetic may differ from the numpy version in the
    last bit at ellipsoid surfaces)."""
    import torch
    X, Y, Z = (int(s) for s in shape_xyz)
    vx, vy, vz = (float(v) for v in voxel_mm)
    params = Ph.ellipsoid_parameters(shape_xyz, voxel_mm, n_ellipsoids, seed)
    xs = (torch.arange(X, dtype=torch.float32, device=device) - (X - 1) / 2) * vx
    ys = (torch.arange(Y, dtype=torch.float32, device=device) - (Y - 1) / 2) * vy
    zs = (torch.arange(Z, dtype=torch.float32, device=device) - (Z - 1) / 2) * vz
    zz, yy, xx = torch.meshgrid(zs, ys, xs, indexing="ij")
    vol = torch.zeros((Z, Y, X), dtype=torch.float32, device=device)
    inside = (xx * xx + yy * yy) <= params["radius"] ** 2
    vol[inside] = params["mu_water"]
    for e in params["ellipsoids"]:
        lo, hi = e["lo"], e["hi"]
        sub = (slice(lo[2], hi[2]), slice(lo[1], hi[1]), slice(lo[0], hi[0]))
        c = torch.tensor(e["centre"], dtype=torch.float32, device=device)
        d = torch.stack([xx[sub] - c[0], yy[sub] - c[1], zz[sub] - c[2]], dim=-1)
        local = d @ torch.tensor(e["R"], dtype=torch.float32, device=device)
        mask = ((local / torch.tensor(e["semi"], dtype=torch.float32, device=device)) ** 2).sum(-1) <= 1.0
        vol[sub] += torch.where(mask, torch.tensor(np.float32(e["mu"]), device=device), torch.zeros((), device=device))
    if texture > 0.0:
        g = torch.Generator(device=device)
        g.manual_seed(seed)
        noise = torch.randn(vol.shape, generator=g, device=device) * texture
        vol = torch.where(inside, vol * (1.0 + noise), vol)
    return vol.contiguous()


@dataclass
class Job:
    name: str
    volume: object        # (Z, Y, X) float32, numpy or torch
    voxel: tuple
    pmats: np.ndarray     # (views, modules, 3, 4)
    channels: int
    rows: int


def c1() -> Job:
    vol = Ph.ellipsoid_phantom((64, 64, 64), (2.0, 2.0, 2.0), 10, seed=1)
    P = G.circular_flat(90, 750.0, 1000.0, G.FlatDetector(128, 128, 1.0, 1.0))
    return Job("64^3 f32 -> 90 x 128^2 circular", vol, (2.0, 2.0, 2.0), P, 128, 128)


def c2_geometry(n_views: int = 360) -> np.ndarray:
    det = G.FlatDetector(512, 512, 0.6, 0.6)
    fan = G.fan_angle(det, 1200.0)
    P = G.circular_flat(360, 750.0, 1200.0, det, angle_range=math.radians(200.0) + fan,
                        rng=np.random.default_rng(2024), jitter_mm=0.5, tilt_deg=0.2)
    if n_views < 360:
        P = np.ascontiguousarray(P[np.linspace(0, 359, n_views).round().astype(int)])
    return P


def c2(n_views: int = 360) -> Job:
    vol = Ph.ellipsoid_phantom((256, 256, 256), (1.0, 1.0, 1.0), 40, seed=2)
    return Job("256^3 f32 -> 360 x 512^2 short scan", vol, (1.0, 1.0, 1.0), c2_geometry(n_views), 512, 512)


def c3_geometry(n_views: int = 1440) -> np.ndarray:
    P = G.helical_cylindrical(1440, 4.0, 570.0, 1040.0, 64, 16, 16, 1.0, -128.0, 128.0)
    if n_views < 1440:
        P = np.ascontiguousarray(P[np.linspace(0, 1439, n_views).round().astype(int)])
    return P


def c3(n_views: int = 1440, device: str = "cuda") -> Job:
    vol = phantom_device((512, 512, 512), (0.5, 0.5, 0.5), 40, seed=3, texture=0.01, device=device)
    return Job("512^3 -> 1440 x 64 x (16 x 16) helical", vol, (0.5, 0.5, 0.5), c3_geometry(n_views), 16, 16)


def c4(device: str = "cuda", n_volumes: int = 64) -> List[Job]:
    rng = np.random.default_rng(4)
    edges = [96, 128, 160, 192, 224, 256]
    dets = [(256, 256), (384, 256), (512, 384), (512, 512), (640, 480), (768, 512)]
    jobs = []
    for i in range(n_volumes):
        shape = tuple(int(e) for e in rng.choice(edges, 3))
        vol = phantom_device(shape, (1.0, 1.0, 1.0), 20, seed=400 + i, device=device)
        n_views = int(rng.integers(30, 361))
        C, R = dets[int(rng.integers(0, len(dets)))]
        pitch = float(rng.uniform(0.5, 1.0))
        P = G.circular_flat(n_views, 750.0, 1000.0, G.FlatDetector(C, R, pitch, pitch),
                            start=float(rng.uniform(0, 2 * math.pi)))
        jobs.append(Job(f"c4[{i}] {shape} -> {n_views} x {C}x{R}", vol, (1.0, 1.0, 1.0), P, C, R))
    return jobs


def c5_base_view() -> np.ndarray:
    """The c2 short-scan geometry's first view on a 256 x 256 detector at 1.2 mm: (modules, 3, 4)."""
    det = G.FlatDetector(256, 256, 1.2, 1.2)
    return G.circular_flat(1, 750.0, 1200.0, det)[0]


def c5_volumes(device: str = "cuda", n: int = 8):
    return [phantom_device((256, 256, 256), (1.0, 1.0, 1.0), 40, seed=500 + i, device=device) for i in range(n)]
