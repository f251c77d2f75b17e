"""B200-native cone-beam forward projector for CTL (drop-in for RayCasterProjector).

The compute path is libctlcu.so (hand-written sm_100a CUDA, C ABI in
include/ctlcu.h); this package is its Python binding and host-side mirror of
CTL's projector interface.
"""
from ._lib import (ACCUM_FP32, ACCUM_FP64, ACCUM_KAHAN, BF16, F16, F32, INTERP_SOFTWARE,  # noqa: F401
                   INTERP_TEXTURE, CtlcuError, LIB_PATH, load)
from .projector import (AcquisitionGeometry, Context, CudaRayCasterProjector, ProjectionData,  # noqa: F401
                        Settings, ViewDimensions, Volume, VoxelVolume)

__all__ = [
    "AcquisitionGeometry", "Context", "CudaRayCasterProjector", "ProjectionData", "Settings",
    "ViewDimensions", "Volume", "VoxelVolume", "CtlcuError", "load", "LIB_PATH",
    "F32", "BF16", "F16", "INTERP_SOFTWARE", "INTERP_TEXTURE", "ACCUM_FP64", "ACCUM_KAHAN", "ACCUM_FP32",
]
