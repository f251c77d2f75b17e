"""DEN file reader/writer (CTL's modules/src/io/den/den_header.h:32-94).

A DEN file is a 6-byte header of three little-endian uint16 (rows, cols,
count) followed by ``count`` row-major ``rows x cols`` arrays, little endian.
CTL stores FullGeometry as count = views*modules 3x4 float64 matrices and
projections as count = views*modules float32 images.
"""
from __future__ import annotations

import numpy as np


def read_den(path, dtype) -> np.ndarray:
    raw = open(path, "rb").read()
    rows, cols, count = (int(v) for v in np.frombuffer(raw[:6], dtype="<u2"))
    data = np.frombuffer(raw[6:], dtype=np.dtype(dtype).newbyteorder("<"))
    if data.size != rows * cols * count:
        raise ValueError(f"{path}: header {rows}x{cols}x{count} does not match {data.size} elements")
    return data.reshape(count, rows, cols).astype(dtype)


def write_den(path, array: np.ndarray) -> None:
    a = np.asarray(array)
    if a.ndim == 2:
        a = a[None]
    count, rows, cols = a.shape
    if max(count, rows, cols) > 0xFFFF:
        raise ValueError("DEN dimensions are limited to 65535")
    with open(path, "wb") as f:
        f.write(np.array([rows, cols, count], dtype="<u2").tobytes())
        f.write(np.ascontiguousarray(a).astype(a.dtype.newbyteorder("<")).tobytes())


def read_full_geometry(path, n_modules: int) -> np.ndarray:
    """FullGeometry as (views, modules, 3, 4) float64."""
    mats = read_den(path, np.float64)
    if mats.shape[1:] != (3, 4) or mats.shape[0] % n_modules:
        raise ValueError(f"{path}: not a 3x4 geometry with {n_modules} modules")
    return mats.reshape(-1, n_modules, 3, 4)
