"""NRRD files of projections (CTL's modules/src/io/nrrd/), through the C ABI.

``save_projections`` writes the header CTL writes for ProjectionData
(io/basetypeio.tpp:342-362, io/nrrd/nrrdfileio.tpp:252-337) and the data,
streamed from device memory or written from host memory; ``header`` and
``load_projections`` read it back (raw, little-endian).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .den import _check, _elem_and_ptr, _handle


def save_projections(ctx, data, path, stream: int = 0) -> None:
    """(views, modules, rows, channels) float32, host or device; ctx may be None for host data."""
    elem, ptr = _elem_and_ptr(data)
    if elem != 4:
        raise ValueError("projections are float32")
    V, M, R, Cn = (int(s) for s in data.shape)
    _check(ctx, L.load().ctlcu_nrrd_write_projections(_handle(ctx), str(path).encode(), C.c_void_p(ptr), V, M, R, Cn,
                                                      C.c_void_p(stream or None)))


def header(path) -> dict:
    """version, sizes (fastest first), element bytes and the data offset."""
    version, n_dims, elem = C.c_uint32(0), C.c_uint32(0), C.c_uint32(0)
    sizes = (C.c_uint32 * 4)()
    offset = C.c_uint64(0)
    L.check(L.load().ctlcu_nrrd_header(str(path).encode(), C.byref(version), C.byref(n_dims), C.byref(sizes),
                                       C.byref(elem), C.byref(offset)))
    return {"version": int(version.value), "sizes": [int(sizes[k]) for k in range(n_dims.value)],
            "elem_bytes": int(elem.value), "offset": int(offset.value)}


def load_projections(ctx, path, out=None, stream: int = 0):
    """A 4-D float32 file (channels, rows, modules, views) as (views, modules, rows, channels)."""
    h = header(path)
    if h["elem_bytes"] != 4 or len(h["sizes"]) != 4:
        raise ValueError(f"{path}: not 4-D float32 projections")
    Cn, R, M, V = h["sizes"]
    if out is None:
        out = np.empty((V, M, R, Cn), np.float32)
    e, ptr = _elem_and_ptr(out)
    _check(ctx, L.load().ctlcu_nrrd_read(_handle(ctx), str(path).encode(), C.c_void_p(ptr),
                                         int(np.prod(tuple(out.shape))) * e, C.c_void_p(stream or None)))
    return out
