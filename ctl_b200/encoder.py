"""Projection matrices of a simple CT system, encoded on the device.

Mirrors CTL's way of describing an acquisition
(acquisition/acquisitionsetup.h, components/*, acquisition/trajectories.h) for
the systems it ships with a single detector, gantry and point source:

    setup = AcquisitionSetup(CylindricalDetector((16, 64), (1.0, 1.0), 40, radians(1.0), 0.2),
                             TubularGantry(1000.0, 550.0), nb_views=10)
    setup.apply_preparation_protocol(HelicalTrajectory(radians(3.6), 1.0))
    P = GeometryEncoder.encode_full_geometry(setup, ctx)      # (10, 40, 3, 4) float64

and hands the whole view loop of GeometryEncoder::encodeFullGeometry
(acquisition/geometryencoder.cpp:67-117) to one device launch
(ctlcu_encode_geometry).  Angles are in radians, lengths in mm, as in CTL.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence, Union

import numpy as np

from . import _lib as L


@dataclass
class CylindricalDetector:
    """CylindricalDetector(nbPixelPerModule, pixelDimensions, nbDetectorModules,
    angulationPerModule, moduleSpacing) (components/cylindricaldetector.h)."""
    nb_pixel_per_module: Sequence[int]
    pixel_dimensions: Sequence[float]
    nb_detector_modules: int
    angulation_per_module: float
    module_spacing: float
    skew_coefficient: float = 0.0


@dataclass
class FlatPanelDetector:
    """FlatPanelDetector(nbPixels, pixelDimensions) (components/flatpaneldetector.h)."""
    nb_pixels: Sequence[int]
    pixel_dimensions: Sequence[float]
    skew_coefficient: float = 0.0


@dataclass
class TubularGantry:
    """TubularGantry(sourceToDetectorDistance, sourceToIsoCenterDistance, rotationAngle,
    pitchPosition, tiltAngle) (components/tubulargantry.h)."""
    source_to_detector_distance: float
    source_to_iso_center_distance: float
    rotation_angle: float = 0.0
    pitch_position: float = 0.0
    tilt_angle: float = 0.0


@dataclass
class CarmGantry:
    """CarmGantry(cArmSpan) (components/carmgantry.h)."""
    c_arm_span: float


@dataclass
class HelicalTrajectory:
    angle_increment: float
    pitch_increment: float = 0.0
    start_pitch: float = 0.0
    start_angle: float = 0.0


@dataclass
class AxialScanTrajectory:
    start_angle: float = 0.0


@dataclass
class WobbleTrajectory:
    angle_span: float
    source_to_isocenter: float
    start_angle: float = 0.0
    wobble_angle: float = np.radians(15.0)
    wobble_freq: float = 1.0


@dataclass
class ShortScanTrajectory:
    source_to_isocenter: float
    start_angle: float = 0.0
    angle_span: float = -np.radians(1.0)  # negative: 180 deg + fan angle


@dataclass
class CirclePlusLineTrajectory:
    angle_span: float
    source_to_isocenter: float
    line_length: float
    fraction_of_views_for_line: float = 0.5
    start_angle: float = 0.0


Detector = Union[CylindricalDetector, FlatPanelDetector]
Gantry = Union[TubularGantry, CarmGantry]
Protocol = Union[HelicalTrajectory, AxialScanTrajectory, WobbleTrajectory, ShortScanTrajectory,
                 CirclePlusLineTrajectory]


class AcquisitionSetup:
    """A system (detector + gantry, point source at the focal spot origin) and
    a number of views, prepared by one protocol."""

    def __init__(self, detector: Detector, gantry: Gantry, nb_views: int):
        self.detector = detector
        self.gantry = gantry
        self.nb_views = int(nb_views)
        self.protocol: Optional[Protocol] = None

    def apply_preparation_protocol(self, protocol: Protocol) -> None:
        tubular = isinstance(protocol, (HelicalTrajectory, AxialScanTrajectory))
        if tubular != isinstance(self.gantry, TubularGantry):
            # the protocol's isApplicableTo() (trajectories.cpp)
            raise ValueError(f"{type(protocol).__name__} does not apply to a {type(self.gantry).__name__}")
        self.protocol = protocol

    def nb_modules(self) -> int:
        d = self.detector
        return 1 if isinstance(d, FlatPanelDetector) else int(d.nb_detector_modules)

    def descriptors(self):
        """The C-ABI descriptors (ctlcu_detector_desc, ctlcu_trajectory_desc)."""
        if self.protocol is None:
            raise ValueError("no preparation protocol applied")
        d, g, p = self.detector, self.gantry, self.protocol
        dd = L.DetectorDesc()
        if isinstance(d, FlatPanelDetector):
            dd.pixels[0], dd.pixels[1] = int(d.nb_pixels[0]), int(d.nb_pixels[1])
            dd.n_modules, dd.flat_panel = 1, 1
        else:
            dd.pixels[0], dd.pixels[1] = int(d.nb_pixel_per_module[0]), int(d.nb_pixel_per_module[1])
            dd.n_modules, dd.flat_panel = int(d.nb_detector_modules), 0
            dd.angulation_rad, dd.module_spacing_mm = float(d.angulation_per_module), float(d.module_spacing)
        dd.pixel_mm[0], dd.pixel_mm[1] = float(d.pixel_dimensions[0]), float(d.pixel_dimensions[1])
        dd.skew = float(d.skew_coefficient)
        t = L.TrajectoryDesc()
        if isinstance(g, TubularGantry):
            t.sdd_mm, t.sid_mm = float(g.source_to_detector_distance), float(g.source_to_iso_center_distance)
            t.pitch_mm, t.tilt_rad = float(g.pitch_position), float(g.tilt_angle)
        else:
            t.carm_span_mm = float(g.c_arm_span)
        if isinstance(p, HelicalTrajectory):
            t.kind = L.TRAJ_HELICAL
            t.angle_increment_rad, t.pitch_increment_mm = float(p.angle_increment), float(p.pitch_increment)
            t.start_pitch_mm, t.start_angle_rad = float(p.start_pitch), float(p.start_angle)
        elif isinstance(p, AxialScanTrajectory):
            t.kind, t.start_angle_rad = L.TRAJ_AXIAL, float(p.start_angle)
        elif isinstance(p, WobbleTrajectory):
            t.kind = L.TRAJ_WOBBLE
            t.angle_span_rad, t.source_to_iso_mm = float(p.angle_span), float(p.source_to_isocenter)
            t.start_angle_rad, t.wobble_angle_rad, t.wobble_freq = (float(p.start_angle), float(p.wobble_angle),
                                                                    float(p.wobble_freq))
        elif isinstance(p, ShortScanTrajectory):
            t.kind = L.TRAJ_SHORT_SCAN
            t.source_to_iso_mm, t.start_angle_rad = float(p.source_to_isocenter), float(p.start_angle)
            t.angle_span_rad = float(p.angle_span)
        else:
            t.kind = L.TRAJ_CIRCLE_PLUS_LINE
            t.angle_span_rad, t.source_to_iso_mm = float(p.angle_span), float(p.source_to_isocenter)
            t.line_length_mm, t.line_fraction = float(p.line_length), float(p.fraction_of_views_for_line)
            t.start_angle_rad = float(p.start_angle)
        return dd, t


class GeometryEncoder:
    @staticmethod
    def encode_full_geometry(setup: AcquisitionSetup, ctx, out=None, stream: int = 0, source_shifts=None):
        """All views' projection matrices, (views, modules, 3, 4) float64.
        `out` may be a device tensor (filled asynchronously on torch's current
        stream, or `stream`) or a numpy array; by default a new numpy array.
        source_shifts: (n, 3) source displacements in mm in the source's frame;
        then the result is (n * views, modules, 3, 4), shift-major."""
        from .projector import _is_cuda, _ptr, torch_stream_handle
        dd, t = setup.descriptors()
        shifts = None if source_shifts is None else np.ascontiguousarray(source_shifts, np.float64).reshape(-1, 3)
        n_sh = 1 if shifts is None else shifts.shape[0]
        shape = (n_sh * setup.nb_views, setup.nb_modules(), 3, 4)
        if out is None:
            out = np.empty(shape, np.float64)
        if tuple(out.shape) != shape:
            raise ValueError(f"out has shape {tuple(out.shape)}, expected {shape}")
        if not stream and _is_cuda(out):
            import torch
            stream = torch_stream_handle(torch.cuda.current_stream(out.device))
        if shifts is None:
            ctx._check(ctx.lib.ctlcu_encode_geometry(ctx.h, C.byref(dd), C.byref(t), setup.nb_views,
                                                     C.c_void_p(_ptr(out)), C.c_void_p(stream or None)))
        else:
            ctx._check(ctx.lib.ctlcu_encode_geometry_shifted(
                ctx.h, C.byref(dd), C.byref(t), setup.nb_views, C.c_void_p(shifts.ctypes.data), n_sh,
                C.c_void_p(_ptr(out)), C.c_void_p(stream or None)))
        return out
