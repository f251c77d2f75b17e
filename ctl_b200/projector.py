"""Host-side interface of the B200 projector, mirroring CTL's projector API.

``CudaRayCasterProjector`` has the method names, settings, parameter keys and
error behaviour of ``CTL::OCL::RayCasterProjector``
(modules/src/projectors/raycasterprojector.h:20-58, raycasterprojector.cpp)
and of the ``AbstractProjector`` interface it implements
(modules/src/projectors/abstractprojector.h:65-144):

  configure(setup)            stores the projection matrices and view dimensions
  project(volume)             -> ProjectionData [view][module][row][channel]
  project_composite(volumes)  sum of the sub-volume projections
  is_linear()                 True
  parameter() / set_parameter(map) with the reference's keys
  to_variant() / from_variant(map)
  settings()                  the Settings object (raysPerPixel, raySampling, ...)
  notifier                    callbacks receiving projectionFinished(view)

``Context`` is the thin, lower-level handle on one device (resident volumes,
device-pointer projection, batches) that the projector and the benchmark use.
Both call the C ABI in libctlcu.so; nothing here computes projections itself.
"""
from __future__ import annotations

import ctypes as C
import logging
import math
from dataclasses import dataclass, field
from typing import Callable, List, Optional, Sequence

import numpy as np

from . import _lib as L

log = logging.getLogger("ctl_b200")


def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _ptr(x) -> int:
    if x is None:
        return 0
    if _is_torch(x):
        return x.data_ptr()
    return x.ctypes.data


def _contig_f64(x):
    if _is_torch(x):
        import torch
        return x.to(torch.float64).contiguous()
    return np.ascontiguousarray(x, dtype=np.float64)


def _contig_f32(x):
    if _is_torch(x):
        import torch
        return x.to(torch.float32).contiguous()
    return np.ascontiguousarray(x, dtype=np.float32)


def _is_cuda(x) -> bool:
    return _is_torch(x) and x.is_cuda


def _check_device_tensor(x, name: str, dtype: str, ndim: int, device: int) -> None:
    """Raise ValueError unless x is a contiguous torch CUDA tensor of `dtype`
    with `ndim` dimensions on CUDA device `device`: a buffer the kernels may
    index by its shape alone."""
    if not _is_cuda(x):
        raise ValueError(f"{name} must be a CUDA tensor")
    if str(x.dtype) != f"torch.{dtype}":
        raise ValueError(f"{name} must be {dtype}, got {x.dtype}")
    if x.dim() != ndim:
        raise ValueError(f"{name} must have {ndim} dimensions, got shape {tuple(x.shape)}")
    if not x.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if x.device.index != device:
        raise ValueError(f"{name} is on cuda:{x.device.index}, the context on cuda:{device}")


def _check_out(out, V: int, M: int, rows: int, channels: int) -> None:
    """A caller-supplied projection buffer must hold exactly [V][M][rows][channels]
    float32 values in that order, or the kernel would write past it."""
    shape = tuple(out.shape)
    want = (V, M, rows, channels)
    if shape != want:
        raise ValueError(f"out must be shaped {want} (views, modules, rows, channels), got {shape}")
    if _is_torch(out):
        if str(out.dtype) != "torch.float32" or not out.is_contiguous():
            raise ValueError("out must be a contiguous float32 tensor")
    elif out.dtype != np.float32 or not out.flags["C_CONTIGUOUS"]:
        raise ValueError("out must be a C-contiguous float32 array")


def torch_stream_handle(stream) -> int:
    """The C-ABI stream argument for a torch CUDA stream.  torch's default
    stream has the handle 0, which the C ABI reads as the context's own
    stream; it is passed as the legacy default stream instead."""
    return stream.cuda_stream or L.STREAM_LEGACY


# ---------------------------------------------------------------------------------------------
# settings, volumes, projection data
# ---------------------------------------------------------------------------------------------

@dataclass
class Settings:
    """RayCasterProjector::Settings (raycasterprojector.h:27-37) plus the B200 options."""
    device_ids: List[int] = field(default_factory=list)
    rays_per_pixel: List[int] = field(default_factory=lambda: [1, 1])
    ray_sampling: float = 0.3
    volume_upsampling: int = 1
    interpolate: bool = True
    interp_mode: int = L.INTERP_SOFTWARE
    accum: int = L.ACCUM_KAHAN
    storage: int = L.F32
    kernel: int = L.KERNEL_AUTO
    # resident copies of recently projected host volumes kept per device by the
    # projector (0: upload every call, as the reference does)
    volume_cache: int = 4
    # launch shape (0 = autotuned for the volume and detector, else the default)
    views_per_block: int = 0
    lanes_x: int = 0
    block_rays: int = 0
    unroll: int = 0

    def to_c(self) -> L.Settings:
        s = L.Settings()
        s.rays_per_pixel[0] = int(self.rays_per_pixel[0])
        s.rays_per_pixel[1] = int(self.rays_per_pixel[1])
        s.ray_sampling = float(self.ray_sampling)
        s.volume_upsampling = int(self.volume_upsampling)
        s.interpolate = 1 if self.interpolate else 0
        s.interp_mode = int(self.interp_mode)
        s.accum = int(self.accum)
        s.kernel = int(self.kernel)
        s.views_per_block = int(self.views_per_block)
        s.lanes_x = int(self.lanes_x)
        s.block_rays = int(self.block_rays)
        s.unroll = int(self.unroll)
        return s

    def launch_shape(self) -> dict:
        return {"views_per_block": self.views_per_block, "lanes_x": self.lanes_x,
                "block_rays": self.block_rays, "unroll": self.unroll}

    @staticmethod
    def optimized_for(smallest_voxel_mm: float, pixel_dims_mm: Sequence[float]) -> "Settings":
        """Settings::optimizedFor (raycasterprojector.cpp:482-521): rays per pixel
        for rectangular pixels, an up-sampling factor for voxels larger than the
        pixels, more rays for voxels smaller than the pixels."""
        ret = Settings()
        xmm, ymm = float(pixel_dims_mm[0]), float(pixel_dims_mm[1])
        if xmm == 0.0 or ymm == 0.0:
            raise RuntimeError("pixel dimensions are singular")
        ratio = xmm / ymm
        broad = ratio > 1.0
        if broad:
            ratio = 1.0 / ratio
        deviation = abs(ratio - 1.0)
        for r in ((1, 2), (1, 3), (1, 4), (2, 3), (3, 4)):
            if abs(ratio - r[0] / r[1]) < deviation:
                deviation = abs(ratio - r[0] / r[1])
                ret.rays_per_pixel = [r[1] if broad else r[0], r[0] if broad else r[1]]
        smallest_pixel = min(xmm / ret.rays_per_pixel[0], ymm / ret.rays_per_pixel[1])
        ret.volume_upsampling = max(int(smallest_voxel_mm / smallest_pixel), 1)
        inc = max(int(smallest_pixel / smallest_voxel_mm), 1)
        ret.rays_per_pixel = [ret.rays_per_pixel[0] * inc, ret.rays_per_pixel[1] * inc]
        return ret


@dataclass
class VoxelVolume:
    """Float32 volume, numpy (Z, Y, X) or torch tensor, x fastest; sizes in mm."""
    data: object
    voxel_size: Sequence[float]
    offset: Sequence[float] = (0.0, 0.0, 0.0)

    def has_data(self) -> bool:
        return self.data is not None and int(np.prod(tuple(self.data.shape))) > 0

    def nb_voxels(self):
        z, y, x = tuple(self.data.shape)
        return int(x), int(y), int(z)

    def smallest_voxel_size(self) -> float:
        return float(min(self.voxel_size))

    def desc(self, dtype: int = L.F32) -> L.VolumeDesc:
        d = L.VolumeDesc()
        nx, ny, nz = self.nb_voxels()
        d.n[0], d.n[1], d.n[2] = nx, ny, nz
        for k in range(3):
            d.voxel_mm[k] = float(self.voxel_size[k])
            d.offset_mm[k] = float(self.offset[k])
        d.dtype = int(dtype)
        return d


@dataclass
class ViewDimensions:
    """SingleViewData::Dimensions: channels, rows, modules."""
    nb_channels: int
    nb_rows: int
    nb_modules: int


@dataclass
class AcquisitionGeometry:
    """What configure() extracts from an AcquisitionSetup: the FullGeometry
    (views x modules projection matrices) and the view dimensions
    (raycasterprojector.cpp:97-107)."""
    pmats: np.ndarray           # (views, modules, 3, 4) float64
    view_dim: ViewDimensions


class ProjectionData:
    """[view][module] images of rows x channels, float32 (projectiondata.h:19-95)."""

    def __init__(self, view_dim: ViewDimensions, data=None):
        self.view_dim = view_dim
        if data is None:
            data = np.zeros((0, view_dim.nb_modules, view_dim.nb_rows, view_dim.nb_channels), np.float32)
        self.data = data

    def nb_views(self) -> int:
        return int(self.data.shape[0])

    def view(self, v):
        return self.data[v]

    def module(self, v, m):
        return self.data[v, m]

    def numpy(self) -> np.ndarray:
        if _is_torch(self.data):
            return self.data.detach().cpu().numpy()
        return np.asarray(self.data)

    def __iadd__(self, other: "ProjectionData"):
        self.data = self.data + other.data
        return self

    def __add__(self, other: "ProjectionData"):
        return ProjectionData(self.view_dim, self.data + other.data)


# ---------------------------------------------------------------------------------------------
# context
# ---------------------------------------------------------------------------------------------

class Volume:
    """A volume resident in device memory (handle on a Context)."""

    def __init__(self, ctx: "Context", handle: int, desc: L.VolumeDesc):
        self.ctx = ctx
        self.handle = handle
        self.desc = desc

    @property
    def nbytes(self) -> int:
        b = C.c_uint64(0)
        self.ctx._check(self.ctx.lib.ctlcu_volume_bytes(self.ctx.h, self.handle, C.byref(b)))
        return int(b.value)

    def release(self) -> None:
        if self.handle:
            self.ctx._check(self.ctx.lib.ctlcu_volume_release(self.ctx.h, self.handle))
            self.handle = 0


class Plan:
    """A captured batch (ctlcu_plan): launch() replays setup + persistent projection."""

    def __init__(self, ctx: "Context", handle, requests):
        self.ctx = ctx
        self.h = handle
        self.requests = list(requests)  # keeps the device tensors alive

    def launch(self, stream: int = 0) -> None:
        self.ctx._check(self.ctx.lib.ctlcu_plan_launch(self.h, C.c_void_p(stream or None)))

    def info(self) -> dict:
        """ctlcu_plan_info: the form the plan kept and both forms' replay times (ms)."""
        form, a, b = C.c_int(0), C.c_float(0), C.c_float(0)
        self.ctx._check(self.ctx.lib.ctlcu_plan_info(self.h, C.byref(form), C.byref(a), C.byref(b)))
        return {"form": "grids" if form.value == L.PLAN_GRIDS else "persistent",
                "ms_persistent": float(a.value), "ms_grids": float(b.value)}

    def close(self) -> None:
        if self.h:
            self.ctx._check(self.ctx.lib.ctlcu_plan_destroy(self.h))
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """One CUDA device: stream, memory budget, resident volumes, projection calls."""

    def __init__(self, device: int = 0):
        self.lib = L.load()
        h = C.c_void_p()
        L.check(self.lib.ctlcu_create(int(device), C.byref(h)))
        self.h = h
        self.device = device

    def close(self) -> None:
        if self.h:
            self.lib.ctlcu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, status: int) -> None:
        L.check(status, self.h)

    # ---- memory ---------------------------------------------------------------------------
    def set_memory_budget(self, nbytes: int) -> None:
        self._check(self.lib.ctlcu_set_memory_budget(self.h, int(nbytes)))

    def memory_used(self) -> int:
        b = C.c_uint64(0)
        self._check(self.lib.ctlcu_memory_used(self.h, C.byref(b)))
        return int(b.value)

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        self._check(self.lib.ctlcu_stream(self.h, C.byref(s)))
        return s.value or 0

    def launches(self) -> int:
        n = C.c_uint64(0)
        self._check(self.lib.ctlcu_launch_count(self.h, C.byref(n)))
        return int(n.value)

    # ---- volumes --------------------------------------------------------------------------
    def set_volume_cache(self, max_volumes: int) -> None:
        """ctlcu_set_volume_cache: keep resident copies of the last max_volumes
        distinct host volumes project_volume saw (0 = upload every call)."""
        self._check(self.lib.ctlcu_set_volume_cache(self.h, int(max_volumes)))

    def volume_cache_stats(self) -> dict:
        hits, misses, resident = C.c_uint64(0), C.c_uint64(0), C.c_uint32(0)
        self._check(self.lib.ctlcu_volume_cache_stats(self.h, C.byref(hits), C.byref(misses), C.byref(resident)))
        return {"hits": int(hits.value), "misses": int(misses.value), "resident": int(resident.value)}

    def volume(self, vol: VoxelVolume, dtype: int = L.F32) -> Volume:
        data = _contig_f32(vol.data)
        desc = vol.desc(dtype)
        h = C.c_uint64(0)
        self._check(self.lib.ctlcu_volume_create(self.h, C.byref(desc), C.c_void_p(_ptr(data)),
                                                 1 if _is_cuda(data) else 0, C.byref(h)))
        return Volume(self, int(h.value), desc)

    # ---- projection -----------------------------------------------------------------------
    @staticmethod
    def _out_like(pmats, V, M, R, Cn):
        if _is_cuda(pmats):
            import torch
            return torch.empty((V, M, R, Cn), dtype=torch.float32, device=pmats.device)
        return np.empty((V, M, R, Cn), dtype=np.float32)

    @staticmethod
    def _stream_for(stream: int, *arrays) -> int:
        """Asynchronous calls on device tensors run on torch's current stream
        unless a stream is given, so torch's caching allocator orders the reuse
        of their memory after our kernels."""
        if stream:
            return stream
        for t in arrays:
            if _is_cuda(t):
                import torch
                return torch_stream_handle(torch.cuda.current_stream(t.device))
        return 0

    def project(self, volume: Volume, pmats, channels: int, rows: int,
                settings: Optional[Settings] = None, out=None, stream: int = 0):
        settings = settings or Settings()
        P = _contig_f64(pmats)
        V, M = int(P.shape[0]), int(P.shape[1])
        if out is None:
            out = self._out_like(P, V, M, rows, channels)
        else:
            _check_out(out, V, M, int(rows), int(channels))
        st = settings.to_c()
        stream = self._stream_for(stream, P, out)
        self._check(self.lib.ctlcu_project(self.h, volume.handle, C.byref(st), C.c_void_p(_ptr(P)), V, M,
                                           int(channels), int(rows), C.c_void_p(_ptr(out)),
                                           C.c_void_p(stream or None)))
        return out

    def project_noalloc(self, volume: Volume, pmats, out, settings: Optional[Settings] = None,
                        stream: int = 0):
        """ctlcu_project_noalloc, for callers that cannot allocate device memory
        during the call: device pmats (V,M,3,4) f64 and out (V,M,R,C) f32; the
        ray geometry goes into the library's static scratch array (at most
        NOALLOC_MAX_VIEW_MODULES view-modules per call).  Nothing is converted
        or copied here (that would allocate), so tensors of the wrong type,
        layout, shape or device raise ValueError instead of reaching the kernel."""
        settings = settings or Settings()
        _check_device_tensor(pmats, "pmats", "float64", 4, self.device)
        _check_device_tensor(out, "out", "float32", 4, self.device)
        if tuple(pmats.shape[2:]) != (3, 4):
            raise ValueError(f"pmats must be shaped (views, modules, 3, 4), got {tuple(pmats.shape)}")
        if tuple(out.shape[:2]) != tuple(pmats.shape[:2]):
            raise ValueError(f"out must be shaped (views, modules, rows, channels) with the views and modules "
                             f"of pmats {tuple(pmats.shape[:2])}, got {tuple(out.shape)}")
        V, M = int(pmats.shape[0]), int(pmats.shape[1])
        R, Ch = int(out.shape[2]), int(out.shape[3])
        st = settings.to_c()
        stream = self._stream_for(stream, pmats, out)
        self._check(self.lib.ctlcu_project_noalloc(self.h, volume.handle, C.byref(st), C.c_void_p(_ptr(pmats)),
                                                   V, M, Ch, R, C.c_void_p(_ptr(out)), C.c_void_p(stream or None)))
        return out

    @staticmethod
    def _inplace_f32(data):
        if _is_torch(data):
            import torch
            if data.dtype != torch.float32 or not data.is_contiguous():
                raise ValueError("data must be a contiguous float32 tensor (changed in place)")
        elif not (isinstance(data, np.ndarray) and data.dtype == np.float32 and data.flags.c_contiguous):
            raise ValueError("data must be a C-contiguous float32 array (changed in place)")
        return data

    def _transform(self, fn, data, i0, stream):
        data = self._inplace_f32(data)
        V = int(data.shape[0])
        per_view = int(np.prod(tuple(data.shape[1:]))) if data.ndim > 1 else 1
        arr = None
        if i0 is not None:
            arr = np.ascontiguousarray(np.broadcast_to(np.asarray(i0, np.float64), (V,)))
        stream = self._stream_for(stream, data)
        self._check(fn(self.h, C.c_void_p(_ptr(data)), V, per_view,
                       C.c_void_p(arr.ctypes.data if arr is not None else None), C.c_void_p(stream or None)))
        return data

    def transform_to_extinction(self, data, i0=None, stream: int = 0):
        """ProjectionData::transformToExtinction: p = log(i0 / p) in place, one i0
        per view (scalar, sequence of views, or None for 1)."""
        return self._transform(self.lib.ctlcu_transform_to_extinction, data, i0, stream)

    def transform_to_intensity(self, data, i0=None, stream: int = 0):
        """ProjectionData::transformToIntensity: p = i0 exp(-p) in place."""
        return self._transform(self.lib.ctlcu_transform_to_intensity, data, i0, stream)

    def average_samples(self, data, n_samples: int, out, low_extinction: bool = False, stream: int = 0):
        """ArealFocalSpotExtension's averaging of n_samples projection sets
        (data: device tensor [sample * views, ...]) into `out` (device, [views, ...])."""
        per = int(out.numel())
        if int(data.numel()) != per * n_samples:
            raise ValueError("data must hold n_samples times the values of out")
        stream = self._stream_for(stream, data, out)
        self._check(self.lib.ctlcu_average_samples(self.h, C.c_void_p(_ptr(data)), int(n_samples), per,
                                                   C.c_void_p(_ptr(out)), 1 if low_extinction else 0,
                                                   C.c_void_p(stream or None)))
        return out

    def combine_linear(self, slope_proj, offset_proj, times, out, stream: int = 0):
        """out[v] = float(times[v]) * slope_proj[v] + offset_proj[v] (device tensors
        [views, ...]): projections of a linear dynamic volume, by linearity."""
        V = int(out.shape[0])
        per_view = int(out.numel()) // V
        t = np.ascontiguousarray(np.broadcast_to(np.asarray(times, np.float64), (V,)))
        stream = self._stream_for(stream, out)
        self._check(self.lib.ctlcu_combine_linear(self.h, C.c_void_p(_ptr(slope_proj)), C.c_void_p(_ptr(offset_proj)),
                                                  C.c_void_p(t.ctypes.data), V, per_view, C.c_void_p(_ptr(out)),
                                                  C.c_void_p(stream or None)))
        return out

    def poisson_noise(self, data, i0_per_module, seed: int, stream: int = 0):
        """PoissonNoiseExtension's noise on extinction data [view][module][rows][channels]
        in place; i0_per_module: photons per pixel of each module."""
        data = self._inplace_f32(data)
        V, M = int(data.shape[0]), int(data.shape[1])
        ppm = int(np.prod(tuple(data.shape[2:])))
        i0 = np.ascontiguousarray(np.broadcast_to(np.asarray(i0_per_module, np.float32), (M,)))
        stream = self._stream_for(stream, data)
        self._check(self.lib.ctlcu_poisson_noise(self.h, C.c_void_p(_ptr(data)), V, M, ppm,
                                                 C.c_void_p(i0.ctypes.data), C.c_uint64(int(seed)),
                                                 C.c_void_p(stream or None)))
        return data

    def detector_saturation(self, data, model: "L.SaturationModel", domain: int, scale=None, stream: int = 0):
        """DetectorSaturationExtension's step on extinction data [view][module][rows][channels]
        in place.  domain: L.SATURATION_EXTINCTION / _PHOTON_COUNT / _INTENSITY; scale: the
        photon count (or count x mean energy) per [view][module] for the last two."""
        data = self._inplace_f32(data)
        V, M = int(data.shape[0]), int(data.shape[1])
        ppm = int(np.prod(tuple(data.shape[2:])))
        arr = None
        if scale is not None:
            arr = np.ascontiguousarray(np.broadcast_to(np.asarray(scale, np.float32), (V, M)))
        stream = self._stream_for(stream, data)
        self._check(self.lib.ctlcu_detector_saturation(self.h, C.c_void_p(_ptr(data)), V, M, ppm, int(domain),
                                                       C.byref(model),
                                                       C.c_void_p(arr.ctypes.data if arr is not None else None),
                                                       C.c_void_p(stream or None)))
        return data

    def project_volume(self, vol: VoxelVolume, pmats, channels: int, rows: int,
                       settings: Optional[Settings] = None, out=None):
        """One-shot: upload, project, release (the reference's per-call semantics)."""
        settings = settings or Settings()
        data = _contig_f32(vol.data)
        P = _contig_f64(pmats)
        V, M = int(P.shape[0]), int(P.shape[1])
        if out is None:
            out = self._out_like(P, V, M, rows, channels)
        else:
            _check_out(out, V, M, int(rows), int(channels))
        desc = vol.desc(settings.storage)
        st = settings.to_c()
        self._check(self.lib.ctlcu_project_volume(self.h, C.byref(desc), C.c_void_p(_ptr(data)), C.byref(st),
                                                  C.c_void_p(_ptr(P)), V, M, int(channels), int(rows),
                                                  C.c_void_p(_ptr(out))))
        return out

    @staticmethod
    def _requests(requests: Sequence[tuple]):
        arr = (L.Request * len(requests))()
        for i, (vol, P, out) in enumerate(requests):
            arr[i].volume = vol.handle
            arr[i].pmats = _ptr(P)
            arr[i].out = _ptr(out)
            arr[i].n_views, arr[i].n_modules = int(P.shape[0]), int(P.shape[1])
            arr[i].rows, arr[i].channels = int(out.shape[2]), int(out.shape[3])
        return arr

    def project_batch(self, requests: Sequence[tuple], settings: Optional[Settings] = None,
                      stream: int = 0) -> None:
        """requests: (Volume, device pmats tensor (V,M,3,4) f64, device out tensor (V,M,R,C) f32).
        All requests' views run in one persistent launch."""
        settings = settings or Settings()
        arr = self._requests(requests)
        st = settings.to_c()
        stream = self._stream_for(stream, *[r[2] for r in requests])
        self._check(self.lib.ctlcu_project_batch(self.h, arr, len(requests), C.byref(st),
                                                 C.c_void_p(stream or None)))

    def plan(self, requests: Sequence[tuple], settings: Optional[Settings] = None,
             form: int = L.PLAN_CHOOSE) -> "Plan":
        """A batch captured once as a CUDA graph; Plan.launch() replays it.  form:
        L.PLAN_CHOOSE (time both forms at creation and keep the faster),
        L.PLAN_PERSISTENT or L.PLAN_GRIDS."""
        settings = settings or Settings()
        arr = self._requests(requests)
        st = settings.to_c()
        h = C.c_void_p()
        self._check(self.lib.ctlcu_plan_create_form(self.h, arr, len(requests), C.byref(st), int(form),
                                                    C.byref(h)))
        return Plan(self, h, requests)

    def sync(self) -> None:
        self._check(self.lib.ctlcu_sync(self.h))

    def count_samples(self, volume: Volume, pmats, channels: int, rows: int,
                      settings: Optional[Settings] = None) -> int:
        settings = settings or Settings()
        P = _contig_f64(pmats)
        n = C.c_uint64(0)
        st = settings.to_c()
        self._check(self.lib.ctlcu_count_samples(self.h, volume.handle, C.byref(st), C.c_void_p(_ptr(P)),
                                                 int(P.shape[0]), int(P.shape[1]), int(channels), int(rows),
                                                 C.byref(n)))
        return int(n.value)

    def autotune(self, volume: Volume, pmats, channels: int, rows: int,
                 settings: Optional[Settings] = None, max_views: int = 8):
        """Time the sample loops on a view subset, then the launch shape of the
        fastest; later KERNEL_AUTO calls with this volume and detector use them.
        Returns (kernel, {loop name: ms with the default shape})."""
        settings = settings or Settings()
        P = _contig_f64(pmats)
        k = C.c_int(0)
        ms = (C.c_float * 3)()
        st = settings.to_c()
        self._check(self.lib.ctlcu_autotune(self.h, volume.handle, C.byref(st), C.c_void_p(_ptr(P)),
                                            int(P.shape[0]), int(P.shape[1]), int(channels), int(rows),
                                            int(max_views), C.byref(k), ms))
        return int(k.value), {"cells": ms[0], "pairs": ms[1], "gather": ms[2]}

    def tuned_settings(self, volume: Volume, n_modules: int, channels: int, rows: int,
                       settings: Optional[Settings] = None) -> Settings:
        """The settings a projection of `volume` onto this detector runs with: the
        sample loop and every launch-shape field resolved (ctlcu_tuned_settings)."""
        settings = settings or Settings()
        st = settings.to_c()
        out = L.Settings()
        self._check(self.lib.ctlcu_tuned_settings(self.h, volume.handle, C.byref(st), int(n_modules),
                                                  int(channels), int(rows), C.byref(out)))
        from dataclasses import replace
        return replace(settings, kernel=out.kernel, views_per_block=out.views_per_block, lanes_x=out.lanes_x,
                       block_rays=out.block_rays, unroll=out.unroll)

    def view_setup(self, pmats):
        P = np.ascontiguousarray(pmats, dtype=np.float64)
        V, M = P.shape[0], P.shape[1]
        qr = np.zeros((V, M, 15))
        src = np.zeros((V, 3))
        self._check(self.lib.ctlcu_view_setup(self.h, C.c_void_p(P.ctypes.data), V, M,
                                              C.c_void_p(qr.ctypes.data), C.c_void_p(src.ctypes.data)))
        return qr, src


class Group:
    """Several devices behind one projection (ctlcu_group): the B200 form of
    RayCasterProjector::Settings::deviceIDs (raycasterprojector.h:30).  One
    context per listed device ordinal (an empty list: every device, as in the
    reference); project_volume gives each device a contiguous block of views
    (ctlcu_split_views) with its own upload of the volume, and its result
    equals a one-device call bit for bit."""

    def __init__(self, devices: Sequence[int] = ()):
        self.lib = L.load()
        ids = [int(d) for d in devices]
        arr = (C.c_int * max(1, len(ids)))(*ids)
        h = C.c_void_p()
        L.check(self.lib.ctlcu_group_create(arr, len(ids), C.byref(h)))
        self.h = h
        self.devices = tuple(ids)

    def size(self) -> int:
        n = C.c_uint32(0)
        L.check_group(self.lib.ctlcu_group_size(self.h, C.byref(n)), self.h)
        return int(n.value)

    def set_volume_cache(self, max_volumes: int) -> None:
        """ctlcu_set_volume_cache on every device's context of the group."""
        for i in range(self.size()):
            ctx = C.c_void_p()
            L.check_group(self.lib.ctlcu_group_context(self.h, i, C.byref(ctx)), self.h)
            L.check(self.lib.ctlcu_set_volume_cache(ctx, int(max_volumes)), ctx)

    def close(self) -> None:
        if self.h:
            self.lib.ctlcu_group_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def project_volume(self, vol: VoxelVolume, pmats, channels: int, rows: int,
                       settings: Optional[Settings] = None, out=None) -> np.ndarray:
        """ctlcu_group_project_volume: host volume, pmats and output."""
        settings = settings or Settings()
        data = np.ascontiguousarray(vol.data, dtype=np.float32)
        P = np.ascontiguousarray(pmats, dtype=np.float64)
        V, M = int(P.shape[0]), int(P.shape[1])
        if out is None:
            out = np.empty((V, M, int(rows), int(channels)), np.float32)
        else:
            _check_out(out, V, M, int(rows), int(channels))
        desc = vol.desc(settings.storage)
        st = settings.to_c()
        L.check_group(self.lib.ctlcu_group_project_volume(
            self.h, C.byref(desc), C.c_void_p(data.ctypes.data), C.byref(st), C.c_void_p(P.ctypes.data), V, M,
            int(channels), int(rows), C.c_void_p(out.ctypes.data)), self.h)
        return out


# ---------------------------------------------------------------------------------------------
# the AbstractProjector mirror
# ---------------------------------------------------------------------------------------------

class CudaRayCasterProjector:
    """Drop-in for CTL::OCL::RayCasterProjector on B200s.

    ``settings().device_ids`` lists the devices a projection is spread over,
    as the reference's deviceIDs (raycasterprojector.h:30; empty: every
    device, raycasterprojector.cpp:449-454).  A list of just the context's
    device (``device``, where the extensions keep their resident volumes)
    projects on that context; any other list goes through a ``Group``."""

    TYPE_ID = 1  # CTL_TYPE_ID(1) of RayCasterProjector (raycasterprojector.h:22)

    def __init__(self, device: int = 0):
        # the reference constructor throws when OpenCL or its kernels are
        # missing (raycasterprojector.cpp:388-422); here loading the library
        # or binding the device raises
        self._settings = Settings()
        self._ctx = Context(device)
        self._group: Optional[Group] = None
        self._geometry: Optional[AcquisitionGeometry] = None
        self.notifier: List[Callable[[int], None]] = []

    def _group_for(self, ids) -> Group:
        """The device group of this id list, rebuilt when the list changes; an
        ordinal that does not exist raises (raycasterprojector.cpp:442-447)."""
        if self._group is None or self._group.devices != tuple(ids):
            if self._group is not None:
                self._group.close()
                self._group = None
            self._group = Group(ids)
        return self._group

    # ---- AbstractProjector ----------------------------------------------------------------
    def configure(self, setup: AcquisitionGeometry) -> None:
        """raycasterprojector.cpp:97-107"""
        P = np.ascontiguousarray(setup.pmats, dtype=np.float64)
        if P.ndim != 4 or P.shape[2:] != (3, 4) or P.shape[1] != setup.view_dim.nb_modules:
            raise ValueError("FullGeometry must be (views, modules, 3, 4) with modules = nbModules")
        self._geometry = AcquisitionGeometry(P, setup.view_dim)

    def project(self, volume: VoxelVolume) -> ProjectionData:
        """raycasterprojector.cpp:139-375.  An invalid volume logs an error and
        returns empty ProjectionData; a device error logs and returns the
        (zero) result, as the reference does."""
        if self._geometry is None:
            raise RuntimeError("CudaRayCasterProjector::project: configure() has not been called")
        vd = self._geometry.view_dim
        ret = ProjectionData(vd)
        if not self._settings.interpolate:
            self._settings.volume_upsampling = 1
        if not volume.has_data():
            log.critical("no or contradictory data in volume object")
            return ret
        if volume.smallest_voxel_size() <= 0.0:
            log.warning("voxel size is zero or negative")
        P = self._geometry.pmats
        # the device list is checked before the projection, outside its error
        # handling: a bad ordinal raises (raycasterprojector.cpp:142, :442-447)
        ids = [int(d) for d in self._settings.device_ids] or list(range(L.device_count()))
        group = self._group_for(ids) if ids != [self._ctx.device] else None
        try:
            if group is not None:
                group.set_volume_cache(self._settings.volume_cache)
                out = group.project_volume(volume, P, vd.nb_channels, vd.nb_rows, self._settings)
            else:
                self._ctx.set_volume_cache(self._settings.volume_cache)
                out = self._ctx.project_volume(volume, P, vd.nb_channels, vd.nb_rows, self._settings)
            ret.data = out
        except L.CtlcuError as e:
            log.critical("ctlcu error: %s", e)
            if e.status == L.ERR_SINGULAR_GEOMETRY:
                pass
            ret.data = np.zeros((P.shape[0], vd.nb_modules, vd.nb_rows, vd.nb_channels), np.float32)
        for v in range(P.shape[0]):
            for cb in self.notifier:
                cb(v)
        return ret

    def project_composite(self, volumes: Sequence[VoxelVolume]) -> ProjectionData:
        """AbstractProjector::projectComposite (abstractprojector.h:99-112)."""
        if len(volumes) == 0:
            raise RuntimeError("AbstractProjector::projectComposite: Volume is empty.")
        ret = self.project(volumes[0])
        for v in volumes[1:]:
            ret += self.project(v)
        return ret

    def is_linear(self) -> bool:
        return True

    # ---- parameters / serialisation (raycasterprojector.cpp:60-91) --------------------------
    def parameter(self) -> dict:
        s = self._settings
        return {
            "Rays per pixel X": int(s.rays_per_pixel[0]),
            "Rays per pixel Y": int(s.rays_per_pixel[1]),
            "Ray sampling step length": float(s.ray_sampling),
            "Volume upsampling factor": int(s.volume_upsampling),
            "Interpolate": bool(s.interpolate),
            "Interpolation mode": "texture" if s.interp_mode == L.INTERP_TEXTURE else "software",
            "Accumulation": {L.ACCUM_FP64: "fp64", L.ACCUM_KAHAN: "kahan", L.ACCUM_FP32: "fp32"}[s.accum],
            "Storage": {L.F32: "f32", L.BF16: "bf16", L.F16: "f16"}[s.storage],
        }

    def set_parameter(self, parameter: dict) -> None:
        m = dict(parameter)
        s = self._settings
        s.rays_per_pixel = [int(m.get("Rays per pixel X", 1)), int(m.get("Rays per pixel Y", 1))]
        s.ray_sampling = float(m.get("Ray sampling step length", 0.3))
        s.volume_upsampling = int(m.get("Volume upsampling factor", 1))
        s.interpolate = bool(m.get("Interpolate", True))
        s.interp_mode = L.INTERP_TEXTURE if m.get("Interpolation mode", "software") == "texture" \
            else L.INTERP_SOFTWARE
        s.accum = {"fp64": L.ACCUM_FP64, "kahan": L.ACCUM_KAHAN, "fp32": L.ACCUM_FP32}[
            m.get("Accumulation", "kahan")]
        s.storage = {"f32": L.F32, "bf16": L.BF16, "f16": L.F16}[m.get("Storage", "f32")]

    def to_variant(self) -> dict:
        return {"type-id": self.TYPE_ID, "#": "CudaRayCasterProjector", "parameters": self.parameter()}

    def from_variant(self, variant: dict) -> None:
        self.set_parameter(variant.get("parameters", {}))

    def settings(self) -> Settings:
        return self._settings

    @property
    def context(self) -> Context:
        return self._ctx
