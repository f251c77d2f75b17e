"""DEN files (CTL's modules/src/io/den/).

A DEN file is a 6-byte header of three little-endian uint16 (rows, cols,
count) followed by ``count`` row-major ``rows x cols`` arrays, with the element
type implied by the file size (den_header.tpp:51-80, den_utils.tpp:8-24).
CTL stores FullGeometry as count = views*modules 3x4 float64 matrices,
projections as count = views*modules float32 images of rows x channels, and
voxel volumes as count = Z slices of Y x X (io/den/denfileio.h:53-68).

``save_*``/``load_*`` go through the C ABI (ctlcu_den_write / ctlcu_den_read):
device tensors stream to and from the file through pinned staging buffers,
host arrays directly.  ``read_den``/``write_den`` are the plain numpy forms.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L

_ELEM = {np.dtype(np.uint8): 1, np.dtype(np.uint16): 2, np.dtype(np.float32): 4, np.dtype(np.float64): 8}
_TYPE = {1: np.uint8, 2: np.uint16, 4: np.float32, 8: np.float64}


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


# ---- through the C ABI (host or device data) ----------------------------------------------

def _handle(ctx):
    return ctx.h if ctx is not None else None


def _check(ctx, status):
    if ctx is not None:
        ctx._check(status)
    else:
        L.check(status)


def _elem_and_ptr(data):
    from .projector import _is_torch, _ptr
    if _is_torch(data):
        import torch
        if not data.is_contiguous():
            raise ValueError("data must be contiguous")
        dt = {torch.uint8: 1, torch.int16: 2, torch.float32: 4, torch.float64: 8}.get(data.dtype)
    else:
        if not data.flags.c_contiguous:
            raise ValueError("data must be C-contiguous")
        dt = _ELEM.get(data.dtype)
    if dt is None:
        raise ValueError(f"DEN holds uint8, uint16, float32 or float64, not {data.dtype}")
    return dt, _ptr(data)


def save(ctx, data, path, rows: int, cols: int, count: int, stream: int = 0) -> None:
    """io::den::save: `count` rows x cols matrices from host or device memory."""
    elem, ptr = _elem_and_ptr(data)
    if rows * cols * count != int(np.prod(tuple(data.shape))):
        raise ValueError("rows x cols x count does not match the data")
    _check(ctx, L.load().ctlcu_den_write(_handle(ctx), str(path).encode(), C.c_void_p(ptr), elem, rows, cols, count,
                                         C.c_void_p(stream or None)))


def header(path):
    """(rows, cols, count), element bytes."""
    dims = (C.c_uint32 * 3)()
    elem = C.c_uint32(0)
    L.check(L.load().ctlcu_den_header(str(path).encode(), C.byref(dims), C.byref(elem)))
    return (int(dims[0]), int(dims[1]), int(dims[2])), int(elem.value)


def load(ctx, path, out=None, first: int = 0, n: int = 0, stream: int = 0):
    """io::den::load of matrices first .. first+n-1 (n = 0: to the end), into `out`
    (host array or device tensor) or a new numpy array of shape (n, rows, cols)."""
    (rows, cols, count), elem = header(path)
    n = n or count - first
    if out is None:
        out = np.empty((n, rows, cols), _TYPE[elem])
    e, ptr = _elem_and_ptr(out)
    if e != elem:
        raise ValueError(f"{path} holds {elem}-byte elements, `out` {e}-byte ones")
    nbytes = int(np.prod(tuple(out.shape))) * e
    _check(ctx, L.load().ctlcu_den_read(_handle(ctx), str(path).encode(), C.c_void_p(ptr), nbytes, first, n,
                                        C.c_void_p(stream or None)))
    return out


def save_projections(ctx, data, path, stream: int = 0) -> None:
    """BaseTypeIO<DenFileIO>::write(ProjectionData): (views, modules, rows, channels) float32."""
    V, M, R, Cn = (int(s) for s in data.shape)
    save(ctx, data, path, R, Cn, V * M, stream)


def load_projections(ctx, path, n_modules: int, out=None, stream: int = 0):
    """BaseTypeIO<DenFileIO>::readProjections: (views, modules, rows, channels) float32."""
    (rows, cols, count), elem = header(path)
    if elem != 4 or count % n_modules:
        raise ValueError(f"{path}: not float32 projections of {n_modules} modules")
    if out is None:
        out = np.empty((count // n_modules, n_modules, rows, cols), np.float32)
    return load(ctx, path, out, 0, count, stream)


def save_full_geometry(ctx, pmats, path) -> None:
    """BaseTypeIO<DenFileIO>::write(FullGeometry): (views, modules, 3, 4) float64."""
    P = np.ascontiguousarray(pmats, np.float64)
    save(ctx, P, path, 3, 4, P.shape[0] * P.shape[1])


def load_full_geometry(ctx, path, n_modules: int) -> np.ndarray:
    """BaseTypeIO<DenFileIO>::readFullGeometry(fileName, nbModules)."""
    (rows, cols, count), elem = header(path)
    if (rows, cols, elem) != (3, 4, 8) or count % n_modules:
        raise ValueError(f"{path}: not a 3x4 float64 geometry with {n_modules} modules")
    out = np.empty((count // n_modules, n_modules, 3, 4))
    return load(ctx, path, out)
