"""Projector extensions that multiply project() calls, done as batched device work.

CTL's extensions wrap a nested projector and call its configure()/project()
once per sub-case (projectors/projectorextension.cpp), and every nested call
re-uploads the volume (projectors/raycasterprojector.cpp:239-269).  With the
volume resident and the geometry encoded on the device, the sub-cases become
one launch each of geometry, projection and reduction:

  ArealFocalSpotExtension (projectors/arealfocalspotextension.cpp:82-160):
    D x D focal-spot samples -> ctlcu_encode_geometry_shifted (all samples' matrices),
    one ctlcu_project over samples x views, ctlcu_average_samples (intensity
    domain, or extinction domain with the low-extinction approximation).
  PoissonNoiseExtension (projectors/poissonnoiseextension.cpp:35-68):
    ctlcu_poisson_noise on the device result.
"""
from __future__ import annotations

from typing import Optional, Sequence, Tuple

import numpy as np

from . import encoder as E
from .projector import Context, Settings, Volume, VoxelVolume


def discretization_grid(nx: int, ny: int):
    """ArealFocalSpotExtension::discretizationGrid: nx x ny points over
    [-1/2, 1/2]^2, x outer and y inner; a single point is the centre."""
    xs = [-0.5 + i / (nx - 1) for i in range(nx)] if nx > 1 else [0.0]
    ys = [-0.5 + j / (ny - 1) for j in range(ny)] if ny > 1 else [0.0]
    return [(x, y) for x in xs for y in ys]


class _Resident:
    """The nested projector's volume, uploaded once and reused by every
    sub-case (and by later project() calls with the same volume object)."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        self._key = None
        self._vol: Optional[Volume] = None

    def get(self, volume, storage: int) -> Volume:
        if isinstance(volume, Volume):
            return volume
        key = (id(volume.data), tuple(volume.data.shape), tuple(volume.voxel_size), tuple(volume.offset), storage)
        if key != self._key:
            if self._vol is not None:
                self._vol.release()
            self._vol = self.ctx.volume(volume, storage)
            self._key = key
        return self._vol

    def release(self):
        if self._vol is not None:
            self._vol.release()
        self._vol, self._key = None, None


class ArealFocalSpotExtension:
    """ArealFocalSpotExtension around the B200 projector.

    configure(setup, focal_spot_size) takes the acquisition (encoder.AcquisitionSetup)
    and the source's focal spot size (width, height) in mm; project(volume) returns
    the (views, modules, rows, channels) extinctions on the device.  A VoxelVolume
    is uploaded on first use and kept resident while the same object is projected
    again (it must not be modified in between; pass a resident Volume to manage
    that explicitly)."""

    def __init__(self, ctx: Context, settings: Optional[Settings] = None,
                 discretization: Tuple[int, int] = (1, 1), low_extinction_approximation: bool = False):
        self.ctx = ctx
        self.settings = settings or Settings()
        self.discretization = tuple(int(d) for d in discretization)
        self.low_extinction_approximation = bool(low_extinction_approximation)
        self._setup: Optional[E.AcquisitionSetup] = None
        self._spot = (0.0, 0.0)
        self._resident = _Resident(ctx)

    def set_discretization(self, nx: int, ny: int) -> None:
        self.discretization = (int(nx), int(ny))

    def enable_low_extinction_approximation(self, enable: bool = True) -> None:
        self.low_extinction_approximation = bool(enable)

    def is_linear(self) -> bool:
        return self.low_extinction_approximation

    def configure(self, setup: E.AcquisitionSetup, focal_spot_size: Sequence[float]) -> None:
        self._setup = setup
        self._spot = (float(focal_spot_size[0]), float(focal_spot_size[1]))

    def source_shifts(self) -> np.ndarray:
        """(samples, 3) source displacements: grid point x spot size (arealfocalspotextension.cpp:116-120)."""
        g = discretization_grid(*self.discretization)
        return np.array([(x * self._spot[0], y * self._spot[1], 0.0) for x, y in g], np.float64)

    def project(self, volume):
        import torch
        if self._setup is None:
            raise RuntimeError("ArealFocalSpotExtension::project: configure() has not been called")
        s = self._setup
        d = s.detector
        C_, R = ((int(d.nb_pixels[0]), int(d.nb_pixels[1])) if isinstance(d, E.FlatPanelDetector)
                 else (int(d.nb_pixel_per_module[0]), int(d.nb_pixel_per_module[1])))
        V, M = s.nb_views, s.nb_modules()
        shifts = self.source_shifts()
        S = shifts.shape[0]
        vol = self._resident.get(volume, self.settings.storage)
        P = torch.empty((S * V, M, 3, 4), dtype=torch.float64, device="cuda")
        E.GeometryEncoder.encode_full_geometry(s, self.ctx, out=P, source_shifts=shifts)
        if S == 1:
            return self.ctx.project(vol, P, C_, R, self.settings)
        sub = self.ctx.project(vol, P, C_, R, self.settings)      # one launch over samples x views
        out = torch.empty((V, M, R, C_), dtype=torch.float32, device="cuda")
        return self.ctx.average_samples(sub, S, out, self.low_extinction_approximation)

    def release(self) -> None:
        self._resident.release()


class PoissonNoiseExtension:
    """PoissonNoiseExtension around a B200 projector or extension (anything with
    project(volume) returning device extinctions [views, modules, rows, channels]).
    photons_per_pixel: i0 per module (RadiationEncoder::photonsPerPixel of the setup)."""

    def __init__(self, nested, photons_per_pixel, fixed_seed: Optional[int] = None):
        if not isinstance(getattr(nested, "ctx", None), Context):
            raise TypeError("the nested projector must be a B200 projector or extension (with a Context)")
        self.nested = nested
        self.ctx = nested.ctx
        self.i0 = np.atleast_1d(np.asarray(photons_per_pixel, np.float32))
        self.fixed_seed = fixed_seed
        self._calls = 0

    def is_linear(self) -> bool:
        return False

    def project(self, volume):
        out = self.nested.project(volume)
        if self.fixed_seed is not None:
            seed = self.fixed_seed + self._calls  # a new draw per call, reproducible per seed
        else:
            seed = int.from_bytes(np.random.bytes(8), "little")
        self._calls += 1
        i0 = np.broadcast_to(self.i0, (int(out.shape[1]),))
        return self.ctx.poisson_noise(out, i0, seed)
