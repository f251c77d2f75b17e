"""Shared helpers for the test suite."""
from __future__ import annotations

import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# Error measure used for every parity statement:
#   |a - b| / max(|b|, 1e-3 * max|b|)
# (the floor keeps grazing rays with near-zero line integrals meaningful).
FLOOR = 1e-3


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    floor = FLOOR * np.abs(b).max() if b.size else 1.0
    den = np.maximum(np.abs(b), floor if floor > 0 else 1e-30)
    return np.abs(a - b) / den


def golden_cases():
    z = np.load(os.path.join(GOLDEN, "projections.npz"))
    meta = json.loads(bytes(z["meta"]).decode())
    out = []
    for m in meta:
        n = m["name"]
        out.append((m, z[n + "__volume"], z[n + "__pmats"], z[n + "__ref"]))
    return out


def golden_geometry():
    return dict(np.load(os.path.join(GOLDEN, "geometry.npz")))


def dequant_bf16(x: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 (round to nearest even) -> float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def dequant_f16(x: np.ndarray) -> np.ndarray:
    return np.asarray(x, dtype=np.float32).astype(np.float16).astype(np.float32)


def uniform_box(n, voxel, mu):
    """A uniform (Z, Y, X) volume of attenuation mu."""
    return np.full((n[2], n[1], n[0]), mu, dtype=np.float32)
