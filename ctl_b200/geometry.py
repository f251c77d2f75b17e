"""Projection-matrix generation (FP64, host side) for the benchmark geometries.

A projection matrix maps world millimetres to detector pixel coordinates,
``P = K R [I | -C]`` normalised so that ``|P[2, :3]| = 1`` and ``det M > 0``
(the convention of CTL's ``ProjectionMatrix::compose`` and ``normalized``,
modules/src/mat/projectionmatrix.cpp:43-48,143-149).  Pixel centres sit at
integer coordinates; channel ``x`` runs along a module's columns and row ``y``
along its rows, as in ``GeometryEncoder::computeIndividualModulePMat``
(modules/src/acquisition/geometryencoder.cpp:299-360).

The arrays returned here are the projector's input: ``(views, modules, 3, 4)``
float64, row major -- the layout of CTL's ``FullGeometry`` flattened.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


def normalized(P: np.ndarray) -> np.ndarray:
    """``ProjectionMatrix::normalized`` (projectionmatrix.cpp:143-149)."""
    denom = np.linalg.norm(P[2, :3])
    denom = math.copysign(denom, np.linalg.det(P[:, :3]))
    return P / denom


def compose(K: np.ndarray, R: np.ndarray, C: np.ndarray) -> np.ndarray:
    """``ProjectionMatrix::compose(K, R, source)`` (projectionmatrix.cpp:43-48)."""
    M = K @ R
    return np.hstack([M, (-M @ C).reshape(3, 1)])


def rot_axis(axis: np.ndarray, angle: float) -> np.ndarray:
    """Rotation matrix about a unit axis (Rodrigues)."""
    a = np.asarray(axis, dtype=np.float64)
    a = a / np.linalg.norm(a)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + math.sin(angle) * K + (1 - math.cos(angle)) * (K @ K)


def intrinsic(focal_mm: float, pitch_x: float, pitch_y: float, cx: float, cy: float) -> np.ndarray:
    return np.array([[focal_mm / pitch_x, 0.0, cx], [0.0, focal_mm / pitch_y, cy], [0.0, 0.0, 1.0]])


def camera_rotation(principal: np.ndarray, up: np.ndarray) -> np.ndarray:
    """World->camera rotation whose rows are (channel dir, row dir, principal ray).

    ``up`` is the world direction the detector rows run against (rows grow
    along ``-up``); the result has determinant +1.
    """
    z = principal / np.linalg.norm(principal)
    y = -(up - np.dot(up, z) * z)
    y /= np.linalg.norm(y)
    x = np.cross(y, z)
    return np.vstack([x, y, z])


@dataclass
class FlatDetector:
    channels: int
    rows: int
    pitch_x: float
    pitch_y: float


def circular_flat(n_views: int, sid: float, sdd: float, det: FlatDetector,
                  angle_range: float = 2 * math.pi, start: float = 0.0,
                  z: float = 0.0, rng: np.random.Generator | None = None,
                  jitter_mm: float = 0.0, tilt_deg: float = 0.0) -> np.ndarray:
    """Circular (or short-scan) cone beam about the world z axis, one flat module.

    With ``rng`` set, each view gets a seeded uniform jitter of +-``jitter_mm``
    on the source and on the detector position and a +-``tilt_deg`` detector
    tilt about each in-plane axis.
    """
    out = np.empty((n_views, 1, 3, 4))
    step = angle_range / n_views
    for v in range(n_views):
        th = start + v * step
        src = np.array([sid * math.cos(th), sid * math.sin(th), z])
        principal = np.array([-math.cos(th), -math.sin(th), 0.0])
        up = np.array([0.0, 0.0, 1.0])
        cx = (det.channels - 1) / 2.0
        cy = (det.rows - 1) / 2.0
        R = camera_rotation(principal, up)
        if rng is not None:
            src = src + rng.uniform(-jitter_mm, jitter_mm, 3)
            dshift = rng.uniform(-jitter_mm, jitter_mm, 2)
            cx += dshift[0] / det.pitch_x
            cy += dshift[1] / det.pitch_y
            tx, ty = np.deg2rad(rng.uniform(-tilt_deg, tilt_deg, 2))
            R = (rot_axis(np.array([1.0, 0, 0]), tx) @ rot_axis(np.array([0, 1.0, 0]), ty)) @ R
        K = intrinsic(sdd, det.pitch_x, det.pitch_y, cx, cy)
        out[v, 0] = normalized(compose(K, R, src))
    return out


def fan_angle(det: FlatDetector, sdd: float) -> float:
    return 2.0 * math.atan(0.5 * det.channels * det.pitch_x / sdd)


def helical_cylindrical(n_views: int, turns: float, sid: float, sdd: float,
                        n_modules: int, mod_channels: int, mod_rows: int,
                        pitch: float, z_start: float, z_end: float) -> np.ndarray:
    """Helical trajectory with a curved detector of flat modules on a cylinder.

    Module ``m`` is a flat ``mod_channels x mod_rows`` panel tangent to the
    cylinder of radius ``sdd`` about the source, rotated in-plane by
    ``(m - (n_modules-1)/2) * mod_channels * pitch / sdd`` -- the layout of
    CTL's ``CylindricalDetector`` (modules/src/components/cylindricaldetector.h:28-33).
    The table moves linearly from ``z_start`` to ``z_end`` over the scan.
    """
    out = np.empty((n_views, n_modules, 3, 4))
    dphi = mod_channels * pitch / sdd
    for v in range(n_views):
        th = 2 * math.pi * turns * v / n_views
        z = z_start + (z_end - z_start) * (v / max(n_views - 1, 1))
        src = np.array([sid * math.cos(th), sid * math.sin(th), z])
        principal = np.array([-math.cos(th), -math.sin(th), 0.0])
        up = np.array([0.0, 0.0, 1.0])
        R0 = camera_rotation(principal, up)
        for m in range(n_modules):
            phi = (m - (n_modules - 1) / 2.0) * dphi
            # rotate the module about the camera's row axis (fan direction)
            Rm = rot_axis(np.array([0.0, 1.0, 0.0]), phi) @ R0
            K = intrinsic(sdd, pitch, pitch, (mod_channels - 1) / 2.0, (mod_rows - 1) / 2.0)
            out[v, m] = normalized(compose(K, Rm, src))
    return out


def perturbed_views(base: np.ndarray, n: int, rng: np.random.Generator,
                    trans_mm: float = 10.0, rot_deg: float = 5.0) -> np.ndarray:
    """Rigid perturbations of one view, as in 2D/3D registration DRR requests.

    Each result is ``P @ T`` with ``T`` a seeded rigid motion of the volume
    (uniform +-``rot_deg`` about each axis, +-``trans_mm`` translation).
    """
    out = np.empty((n,) + base.shape)
    for i in range(n):
        ax = np.deg2rad(rng.uniform(-rot_deg, rot_deg, 3))
        Rr = rot_axis(np.array([1.0, 0, 0]), ax[0]) @ rot_axis(np.array([0, 1.0, 0]), ax[1]) \
            @ rot_axis(np.array([0, 0, 1.0]), ax[2])
        T = np.eye(4)
        T[:3, :3] = Rr
        T[:3, 3] = rng.uniform(-trans_mm, trans_mm, 3)
        for m in range(base.shape[0]):
            out[i, m] = normalized(base[m] @ T)
    return out
