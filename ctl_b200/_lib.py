"""ctypes binding of libctlcu.so (include/ctlcu.h).

The library is loaded from this package directory.  There is no fallback: if
it is missing or fails to load, every projector call raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libctlcu.so")
ABI_VERSION = 2  # CTLCU_ABI_VERSION of include/ctlcu.h these bindings follow

OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_INVALID_HANDLE = 2
ERR_OUT_OF_MEMORY = 3
ERR_CUDA = 4
ERR_NO_DEVICE = 5
ERR_SINGULAR_GEOMETRY = 6
ERR_TIMEOUT = 7
ERR_BUSY = 8

F32, BF16, F16 = 0, 1, 2
INTERP_SOFTWARE, INTERP_TEXTURE = 0, 1
ACCUM_FP64, ACCUM_KAHAN, ACCUM_FP32 = 0, 1, 2
KERNEL_AUTO, KERNEL_GATHER, KERNEL_CELLS, KERNEL_PAIRS = 0, 1, 2, 3
# cudaStreamLegacy: the handle of the legacy default stream.  A NULL stream
# argument means the context's own (non-blocking) stream, so work ordered on
# the default stream (torch's default) must name it with this handle.
STREAM_LEGACY = 1
NOALLOC_MAX_VIEW_MODULES = 4096
PLAN_CHOOSE, PLAN_PERSISTENT, PLAN_GRIDS = -1, 0, 1  # ctlcu_plan_form  # scratch entries of ctlcu_project_noalloc

STATUS_NAMES = {
    OK: "OK", ERR_INVALID_ARGUMENT: "INVALID_ARGUMENT", ERR_INVALID_HANDLE: "INVALID_HANDLE",
    ERR_OUT_OF_MEMORY: "OUT_OF_MEMORY", ERR_CUDA: "CUDA", ERR_NO_DEVICE: "NO_DEVICE",
    ERR_SINGULAR_GEOMETRY: "SINGULAR_GEOMETRY", ERR_TIMEOUT: "TIMEOUT", ERR_BUSY: "BUSY",
}


class VolumeDesc(C.Structure):
    _fields_ = [("n", C.c_uint32 * 3), ("voxel_mm", C.c_float * 3), ("offset_mm", C.c_float * 3),
                ("dtype", C.c_int32)]


class Settings(C.Structure):
    _fields_ = [("rays_per_pixel", C.c_uint32 * 2), ("ray_sampling", C.c_float),
                ("volume_upsampling", C.c_uint32), ("interpolate", C.c_int32),
                ("interp_mode", C.c_int32), ("accum", C.c_int32), ("kernel", C.c_int32),
                ("views_per_block", C.c_int32), ("lanes_x", C.c_int32), ("block_rays", C.c_int32),
                ("unroll", C.c_int32)]


TRAJ_HELICAL, TRAJ_AXIAL, TRAJ_WOBBLE, TRAJ_SHORT_SCAN, TRAJ_CIRCLE_PLUS_LINE = 0, 1, 2, 3, 4


class DetectorDesc(C.Structure):
    _fields_ = [("pixels", C.c_uint32 * 2), ("pixel_mm", C.c_double * 2), ("n_modules", C.c_uint32),
                ("flat_panel", C.c_int32), ("angulation_rad", C.c_double), ("module_spacing_mm", C.c_double),
                ("skew", C.c_double)]


class TrajectoryDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("reserved", C.c_int32),
                ("sdd_mm", C.c_double), ("sid_mm", C.c_double), ("pitch_mm", C.c_double), ("tilt_rad", C.c_double),
                ("angle_increment_rad", C.c_double), ("pitch_increment_mm", C.c_double),
                ("start_pitch_mm", C.c_double), ("start_angle_rad", C.c_double),
                ("carm_span_mm", C.c_double), ("source_to_iso_mm", C.c_double), ("angle_span_rad", C.c_double),
                ("wobble_angle_rad", C.c_double), ("wobble_freq", C.c_double),
                ("line_length_mm", C.c_double), ("line_fraction", C.c_double)]


SATURATION_LINEAR, SATURATION_SPLINE = 0, 1
SATURATION_EXTINCTION, SATURATION_PHOTON_COUNT, SATURATION_INTENSITY = 0, 1, 2


class SaturationModel(C.Structure):
    _fields_ = [("kind", C.c_int32), ("a", C.c_float), ("b", C.c_float), ("soft_a", C.c_float),
                ("soft_b", C.c_float)]


class Request(C.Structure):
    _fields_ = [("volume", C.c_uint64), ("pmats", C.c_void_p), ("out", C.c_void_p),
                ("n_views", C.c_uint32), ("n_modules", C.c_uint32), ("channels", C.c_uint32),
                ("rows", C.c_uint32)]


# (name, restype, argtypes) of every entry point declared in include/ctlcu.h
SIGNATURES = [
    ("ctlcu_abi_version", C.c_int, []),
    ("ctlcu_settings_default", Settings, []),
    ("ctlcu_create", C.c_int, [C.c_int, C.POINTER(C.c_void_p)]),
    ("ctlcu_destroy", C.c_int, [C.c_void_p]),
    ("ctlcu_last_error", C.c_char_p, [C.c_void_p]),
    ("ctlcu_set_memory_budget", C.c_int, [C.c_void_p, C.c_uint64]),
    ("ctlcu_memory_used", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    ("ctlcu_stream", C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    ("ctlcu_volume_create", C.c_int, [C.c_void_p, C.POINTER(VolumeDesc), C.c_void_p, C.c_int,
                                      C.POINTER(C.c_uint64)]),
    ("ctlcu_volume_release", C.c_int, [C.c_void_p, C.c_uint64]),
    ("ctlcu_volume_bytes", C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.c_uint64)]),
    ("ctlcu_set_volume_cache", C.c_int, [C.c_void_p, C.c_uint32]),
    ("ctlcu_volume_cache_stats", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                           C.POINTER(C.c_uint32)]),
    ("ctlcu_project", C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(Settings), C.c_void_p, C.c_uint32,
                                C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("ctlcu_project_noalloc", C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(Settings), C.c_void_p, C.c_uint32,
                                        C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("ctlcu_project_volume", C.c_int, [C.c_void_p, C.POINTER(VolumeDesc), C.c_void_p, C.POINTER(Settings),
                                       C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                       C.c_void_p]),
    ("ctlcu_project_batch", C.c_int, [C.c_void_p, C.POINTER(Request), C.c_uint32, C.POINTER(Settings),
                                      C.c_void_p]),
    ("ctlcu_plan_create", C.c_int, [C.c_void_p, C.POINTER(Request), C.c_uint32, C.POINTER(Settings),
                                    C.POINTER(C.c_void_p)]),
    ("ctlcu_plan_launch", C.c_int, [C.c_void_p, C.c_void_p]),
    ("ctlcu_plan_destroy", C.c_int, [C.c_void_p]),
    ("ctlcu_plan_info", C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    ("ctlcu_plan_create_form", C.c_int, [C.c_void_p, C.POINTER(Request), C.c_uint32, C.POINTER(Settings), C.c_int,
                                         C.POINTER(C.c_void_p)]),
    ("ctlcu_sync", C.c_int, [C.c_void_p]),
    ("ctlcu_count_samples", C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(Settings), C.c_void_p, C.c_uint32,
                                      C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint64)]),
    ("ctlcu_autotune", C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(Settings), C.c_void_p, C.c_uint32,
                                 C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.POINTER(C.c_int),
                                 C.POINTER(C.c_float)]),
    ("ctlcu_tuned_settings", C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(Settings), C.c_uint32, C.c_uint32,
                                       C.c_uint32, C.POINTER(Settings)]),
    ("ctlcu_view_setup", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p,
                                   C.c_void_p]),
    ("ctlcu_launch_count", C.c_int, [C.c_void_p, C.POINTER(C.c_uint64)]),
    ("ctlcu_encode_geometry", C.c_int, [C.c_void_p, C.POINTER(DetectorDesc), C.POINTER(TrajectoryDesc), C.c_uint32,
                                        C.c_void_p, C.c_void_p]),
    ("ctlcu_transform_to_extinction", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_void_p,
                                                C.c_void_p]),
    ("ctlcu_transform_to_intensity", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_void_p,
                                               C.c_void_p]),
    ("ctlcu_poisson_noise", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p,
                                      C.c_uint64, C.c_void_p]),
    ("ctlcu_encode_geometry_shifted", C.c_int, [C.c_void_p, C.POINTER(DetectorDesc), C.POINTER(TrajectoryDesc),
                                                C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]),
    ("ctlcu_average_samples", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_void_p, C.c_int,
                                        C.c_void_p]),
    ("ctlcu_combine_linear", C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64,
                                       C.c_void_p, C.c_void_p]),
    ("ctlcu_spectral_combine", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint64, C.c_void_p,
                                         C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]),
    ("ctlcu_detector_saturation", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint64, C.c_int32,
                                            C.POINTER(SaturationModel), C.c_void_p, C.c_void_p]),
    ("ctlcu_spectral_combine_noisy", C.c_int, [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
                                               C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32,
                                               C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p]),
    ("ctlcu_den_write", C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32,
                                  C.c_uint32, C.c_void_p]),
    ("ctlcu_den_header", C.c_int, [C.c_char_p, C.POINTER(C.c_uint32 * 3), C.POINTER(C.c_uint32)]),
    ("ctlcu_nrrd_write_projections", C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p, C.c_uint32, C.c_uint32,
                                               C.c_uint32, C.c_uint32, C.c_void_p]),
    ("ctlcu_nrrd_header", C.c_int, [C.c_char_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                    C.POINTER(C.c_uint32 * 4), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)]),
    ("ctlcu_nrrd_read", C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p, C.c_uint64, C.c_void_p]),
    ("ctlcu_den_read", C.c_int, [C.c_void_p, C.c_char_p, C.c_void_p, C.c_uint64, C.c_uint32, C.c_uint32,
                                 C.c_void_p]),
    ("ctlcu_device_count", C.c_int, [C.POINTER(C.c_int)]),
    ("ctlcu_group_create", C.c_int, [C.POINTER(C.c_int), C.c_uint32, C.POINTER(C.c_void_p)]),
    ("ctlcu_group_destroy", C.c_int, [C.c_void_p]),
    ("ctlcu_group_last_error", C.c_char_p, [C.c_void_p]),
    ("ctlcu_group_size", C.c_int, [C.c_void_p, C.POINTER(C.c_uint32)]),
    ("ctlcu_group_context", C.c_int, [C.c_void_p, C.c_uint32, C.POINTER(C.c_void_p)]),
    ("ctlcu_group_project_volume", C.c_int, [C.c_void_p, C.POINTER(VolumeDesc), C.c_void_p, C.POINTER(Settings),
                                             C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                             C.c_void_p]),
    ("ctlcu_split_views", C.c_int, [C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32)]),
]

_lib = None


def load() -> C.CDLL:
    """Load libctlcu.so and declare its signatures (raises if it is not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run `python -m ctl_b200.build`")
        lib = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        if lib.ctlcu_abi_version() != ABI_VERSION:
            raise ImportError(f"{LIB_PATH} has ABI version {lib.ctlcu_abi_version()}, these bindings "
                              f"expect {ABI_VERSION}; rebuild with `python -m ctl_b200.build`")
        _lib = lib
    return _lib


class CtlcuError(RuntimeError):
    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")


def check(status: int, ctx=None) -> None:
    if status != OK:
        msg = load().ctlcu_last_error(ctx).decode() if ctx else ""
        raise CtlcuError(status, msg)


def check_group(status: int, group) -> None:
    if status != OK:
        raise CtlcuError(status, load().ctlcu_group_last_error(group).decode())


def device_count() -> int:
    """ctlcu_device_count: CUDA devices this process sees."""
    n = C.c_int(0)
    check(load().ctlcu_device_count(C.byref(n)))
    return int(n.value)


def split_views(n_views: int, n_parts: int) -> list:
    """ctlcu_split_views: the first view of each of n_parts contiguous blocks,
    plus n_views at the end (n_parts + 1 entries)."""
    first = (C.c_uint32 * (n_parts + 1))()
    check(load().ctlcu_split_views(int(n_views), int(n_parts), first))
    return list(first)
