"""Seeded synthetic volumes: a water cylinder with additive random ellipsoids.

Volumes are float32, x fastest in memory (index ``z*X*Y + y*X + x``, CTL's
``VoxelVolume`` layout, modules/src/img/voxelvolume.tpp:310-335), returned as
numpy arrays of shape ``(Z, Y, X)``.  Attenuation is in 1/mm.
"""
from __future__ import annotations

import numpy as np


def ellipsoid_parameters(shape_xyz, voxel_mm, n_ellipsoids: int, seed: int) -> dict:
    """The seeded phantom description: water cylinder (axis z, radius 45% of
    the smaller in-plane extent, mu 0.02 /mm) and ellipsoids with semi-axes
    4-25 mm, random rotation and attenuation uniform in 0.005-0.05 /mm, each
    with its voxel bounding box.  Returns the generator too, positioned for the
    texture noise draw."""
    X, Y, Z = (int(s) for s in shape_xyz)
    vx, vy, vz = (float(v) for v in voxel_mm)
    rng = np.random.default_rng(seed)
    radius = 0.45 * min(X * vx, Y * vy)
    ells = []
    for _ in range(n_ellipsoids):
        semi = rng.uniform(4.0, 25.0, 3)
        # centre within the cylinder, away from its wall
        r = rng.uniform(0.0, max(radius - semi.max(), 0.0))
        phi = rng.uniform(0, 2 * np.pi)
        cz = rng.uniform(-0.4, 0.4) * Z * vz
        centre = np.array([r * np.cos(phi), r * np.sin(phi), cz])
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        w, a, b, c = q
        R = np.array([[1 - 2 * (b * b + c * c), 2 * (a * b - c * w), 2 * (a * c + b * w)],
                      [2 * (a * b + c * w), 1 - 2 * (a * a + c * c), 2 * (b * c - a * w)],
                      [2 * (a * c - b * w), 2 * (b * c + a * w), 1 - 2 * (a * a + b * b)]])
        mu = rng.uniform(0.005, 0.05)
        ext = semi.max()
        lo = [max(int(np.floor(((centre[k] - ext) / v) + (n - 1) / 2)), 0) for k, v, n in
              zip(range(3), (vx, vy, vz), (X, Y, Z))]
        hi = [min(int(np.ceil(((centre[k] + ext) / v) + (n - 1) / 2)) + 1, n) for k, v, n in
              zip(range(3), (vx, vy, vz), (X, Y, Z))]
        if any(h <= l for l, h in zip(lo, hi)):
            continue
        ells.append(dict(centre=centre, R=R, semi=semi, mu=mu, lo=lo, hi=hi))
    return dict(radius=radius, mu_water=0.02, ellipsoids=ells, rng=rng)


def ellipsoid_phantom(shape_xyz, voxel_mm, n_ellipsoids: int, seed: int,
                      mu_water: float = 0.02, texture: float = 0.0) -> np.ndarray:
    """Water cylinder plus ``n_ellipsoids`` additive ellipsoids (see
    ellipsoid_parameters); ``texture`` adds seeded Gaussian noise with that
    relative standard deviation inside the cylinder."""
    X, Y, Z = (int(s) for s in shape_xyz)
    vx, vy, vz = (float(v) for v in voxel_mm)
    p = ellipsoid_parameters(shape_xyz, voxel_mm, n_ellipsoids, seed)
    xs = (np.arange(X, dtype=np.float32) - (X - 1) / 2) * vx
    ys = (np.arange(Y, dtype=np.float32) - (Y - 1) / 2) * vy
    zs = (np.arange(Z, dtype=np.float32) - (Z - 1) / 2) * vz
    zz, yy, xx = np.meshgrid(zs, ys, xs, indexing="ij")
    vol = np.zeros((Z, Y, X), dtype=np.float32)
    inside = (xx * xx + yy * yy) <= p["radius"] * p["radius"]
    vol[inside] = mu_water
    for e in p["ellipsoids"]:
        lo, hi = e["lo"], e["hi"]
        sub = (slice(lo[2], hi[2]), slice(lo[1], hi[1]), slice(lo[0], hi[0]))
        d = np.stack([xx[sub] - e["centre"][0], yy[sub] - e["centre"][1], zz[sub] - e["centre"][2]], axis=-1)
        local = d @ e["R"]  # coordinates in the ellipsoid frame
        mask = ((local / e["semi"]) ** 2).sum(axis=-1) <= 1.0
        vol[sub][mask] += np.float32(e["mu"])
    if texture > 0.0:
        noise = p["rng"].standard_normal(vol.shape, dtype=np.float32) * np.float32(texture)
        vol = np.where(inside, vol * (1.0 + noise), vol).astype(np.float32)
    return np.ascontiguousarray(vol)
