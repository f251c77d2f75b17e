"""Test-only checkers for the CUDA projector.

``project_fp64`` runs the FP64 C restatement (liboracle.so); ``project_ref``
runs the reference's own kernel and matrix code compiled for the CPU
(_ref/libctlref.so, built only where the reference sources are present).
Nothing in the product package imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))


class _Volume(C.Structure):
    _fields_ = [("n", C.c_longlong * 3), ("voxel_mm", C.c_float * 3), ("offset_mm", C.c_float * 3)]


class _Settings(C.Structure):
    _fields_ = [("rays_per_pixel", C.c_uint * 2), ("ray_sampling", C.c_float),
                ("volume_upsampling", C.c_uint), ("interpolate", C.c_int)]


def build(with_ref: bool = True) -> None:
    """Compile liboracle.so, and _ref/libctlref.so where the reference sources
    are present (the Makefile's REF, overridable by CTL_REFERENCE_DIR)."""
    subprocess.run(["make", "-s", "-C", _HERE, "all"], check=True)
    if with_ref:
        subprocess.run(["make", "-s", "-C", _HERE, "ref-if-present"], check=True)


_libs: dict = {}


def _lib(name: str):
    if name not in _libs:
        path = os.path.join(_HERE, name)
        if not os.path.exists(path):
            if name == "liboracle.so":
                build(with_ref=False)
            else:
                raise FileNotFoundError(f"{path} is not built (needs the reference sources)")
        lib = C.CDLL(path)
        _libs[name] = lib
    return _libs[name]


def ref_available() -> bool:
    return os.path.exists(os.path.join(_HERE, "_ref", "libctlref.so"))


def _structs(shape_zyx, voxel_mm, offset_mm, rays, ray_sampling, upsampling, interpolate):
    vd = _Volume()
    vd.n[0], vd.n[1], vd.n[2] = int(shape_zyx[2]), int(shape_zyx[1]), int(shape_zyx[0])
    for k in range(3):
        vd.voxel_mm[k] = float(voxel_mm[k])
        vd.offset_mm[k] = float(offset_mm[k])
    st = _Settings()
    st.rays_per_pixel[0], st.rays_per_pixel[1] = int(rays[0]), int(rays[1])
    st.ray_sampling = float(ray_sampling)
    st.volume_upsampling = int(upsampling)
    st.interpolate = int(bool(interpolate))
    return vd, st


def _project(which, volume, voxel_mm, pmats, channels, rows, offset_mm=(0, 0, 0), rays=(1, 1),
             ray_sampling=0.3, upsampling=1, interpolate=True, threads=None):
    vol = np.ascontiguousarray(volume, dtype=np.float32)
    P = np.ascontiguousarray(pmats, dtype=np.float64)
    V, M = P.shape[0], P.shape[1]
    out = np.zeros((V, M, rows, channels), dtype=np.float32)
    vd, st = _structs(vol.shape, voxel_mm, offset_mm, rays, ray_sampling, upsampling, interpolate)
    threads = threads or os.cpu_count() or 1
    fp = C.POINTER(C.c_float)
    dp = C.POINTER(C.c_double)
    if which == "fp64":
        lib = _lib("liboracle.so")
        count = C.c_ulonglong(0)
        rc = lib.oracle_project(vol.ctypes.data_as(fp), C.byref(vd), C.byref(st), P.ctypes.data_as(dp),
                                C.c_uint(V), C.c_uint(M), C.c_uint(channels), C.c_uint(rows),
                                out.ctypes.data_as(fp), C.byref(count), C.c_int(threads))
        if rc:
            raise ValueError(f"oracle_project failed ({rc})")
        return out, int(count.value)
    lib = _lib(os.path.join("_ref", "libctlref.so"))
    rc = lib.ctlref_project(vol.ctypes.data_as(fp), C.byref(vd), C.byref(st), P.ctypes.data_as(dp),
                            C.c_uint(V), C.c_uint(M), C.c_uint(channels), C.c_uint(rows),
                            out.ctypes.data_as(fp), C.c_int(threads))
    if rc:
        raise ValueError(f"ctlref_project failed ({rc})")
    return out


def project_fp64(*args, **kw):
    """FP64 oracle.  Returns (projections [V, M, rows, channels], sample count)."""
    return _project("fp64", *args, **kw)


def project_ref(*args, **kw):
    """Reference kernel compiled for the CPU.  Returns projections [V, M, rows, channels]."""
    return _project("ref", *args, **kw)


def view_setup(pmats, which="fp64"):
    """Per (view, module) packed QR (15 doubles) and per-view source positions."""
    P = np.ascontiguousarray(pmats, dtype=np.float64)
    V, M = P.shape[0], P.shape[1]
    qr = np.zeros((V, M, 15))
    src = np.zeros((V, 3))
    dp = C.POINTER(C.c_double)
    if which == "fp64":
        _lib("liboracle.so").oracle_view_setup(P.ctypes.data_as(dp), C.c_uint(V), C.c_uint(M),
                                               qr.ctypes.data_as(dp), src.ctypes.data_as(dp))
    else:
        _lib(os.path.join("_ref", "libctlref.so")).ctlref_view_setup(
            P.ctypes.data_as(dp), C.c_uint(V), C.c_uint(M), qr.ctypes.data_as(dp), src.ctypes.data_as(dp))
    return qr, src


def poisson_noise(extinction, i0_per_module, seed):
    """The device noise algorithm restated on the CPU (postops_oracle.c):
    returns (noisy extinction, noisy counts), both [V, M, rows, channels]."""
    x = np.array(extinction, dtype=np.float32, copy=True, order="C")
    V, M = x.shape[0], x.shape[1]
    ppm = int(np.prod(x.shape[2:]))
    i0 = np.ascontiguousarray(i0_per_module, dtype=np.float32)
    counts = np.empty_like(x)
    fp = C.POINTER(C.c_float)
    _lib("liboracle.so").oracle_poisson_noise(x.ctypes.data_as(fp), C.c_uint(V), C.c_uint(M), C.c_uint(ppm),
                                              i0.ctypes.data_as(fp), C.c_uint64(seed), counts.ctypes.data_as(fp))
    return x, counts


def poisson_draws(lam, seed, view=0):
    """Draws of the device sampler (one counter stream per entry) for the means `lam`."""
    lam = np.ascontiguousarray(lam, dtype=np.float64).ravel()
    out = np.empty(lam.size, np.float32)
    _lib("liboracle.so").oracle_poisson_draws(lam.ctypes.data_as(C.POINTER(C.c_double)), C.c_uint64(lam.size),
                                              C.c_uint64(seed), C.c_uint(view),
                                              out.ctypes.data_as(C.POINTER(C.c_float)))
    return out


def poisson_noise_reference(extinction, i0_per_module, seed):
    """The reference's noise step with its own mt19937_64 and std:: distributions
    (poisson_ref.cpp): noisy extinction [V, M, rows, channels]."""
    x = np.array(extinction, dtype=np.float32, copy=True, order="C")
    V, M = x.shape[0], x.shape[1]
    ppm = int(np.prod(x.shape[2:]))
    i0 = np.ascontiguousarray(i0_per_module, dtype=np.float32)
    fp = C.POINTER(C.c_float)
    path = os.path.join(_HERE, "libpoissonref.so")
    if not os.path.exists(path):
        build(with_ref=False)
    C.CDLL(path).ref_poisson_noise(x.ctypes.data_as(fp), C.c_uint(V), C.c_uint(M), C.c_uint(ppm),
                                   i0.ctypes.data_as(fp), C.c_uint(seed))
    return x


def saturation_value(x, kind, a, b, soft_a=0.0, soft_b=0.0):
    """DetectorSaturationLinearModel::valueAt / DetectorSaturationSplineModel::valueAt and
    spline1/spline2 (models/detectorsaturationmodels.cpp:27-35, :108-127, :294-307), FP32,
    one rounding per operation in the reference's order."""
    f = np.float32
    x = np.asarray(x, np.float32)
    a, b, sa, sb = f(a), f(b), f(soft_a), f(soft_b)
    if kind == 0:
        return np.where(x < a, a, np.where(x > b, b, x)).astype(np.float32)
    s1s, s1e, s2s, s2e = f(a - sa), f(a + sa), f(b - sb), f(b + sb)
    with np.errstate(over="ignore", invalid="ignore"):
        sp1 = (f(1.0) / (f(4.0) * sa)) * (x * x) - (s1s / (f(2.0) * sa)) * x + (s1e * s1e) / (f(4.0) * sa)
        sp2 = (f(-1.0) / (f(4.0) * sb)) * (x * x) + (s2e / (f(2.0) * sb)) * x - (s2s * s2s) / (f(4.0) * sb)
    out = np.where(x < s1s, a, np.where(x < s1e, sp1, np.where(x < s2s, x, np.where(x < s2e, sp2, b))))
    return out.astype(np.float32)


def detector_saturation(extinction, kind, a, b, soft_a, soft_b, domain, scale=None):
    """DetectorSaturationExtension::processExtinctions / processCounts / processIntensities
    (projectors/detectorsaturationextension.cpp:118-226) on [V, M, ...] extinctions, FP32:
    domain 0 applies the model to the extinctions; 1 and 2 to scale[v][m] * exp(-p), then
    p = log(scale / value).  scale: the photon count (1) or count x mean energy (2)."""
    p = np.array(extinction, dtype=np.float32, copy=True)
    if domain == 0:
        return saturation_value(p, kind, a, b, soft_a, soft_b)
    s = np.asarray(scale, np.float32).reshape(p.shape[:2] + (1,) * (p.ndim - 2))
    with np.errstate(divide="ignore", invalid="ignore"):
        x = saturation_value((s * np.exp(-p)).astype(np.float32), kind, a, b, soft_a, soft_b)
        return np.log((s / x).astype(np.float32)).astype(np.float32)
