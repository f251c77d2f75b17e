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
  DynamicProjectorExtension over a LinearDynamicVolume: two projections and
    ctlcu_combine_linear.
  SpectralEffectsExtension: one batched projection of the material densities and
    ctlcu_spectral_combine (linear), or ctlcu_spectral_combine_noisy around a
    nested PoissonNoiseExtension.
  DetectorSaturationExtension (projectors/detectorsaturationextension.cpp:96-226):
    ctlcu_detector_saturation on the device result.
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
        self._data = None  # the uploaded array, held so that its id stays unique while cached
        self._vol: Optional[Volume] = None

    def get(self, volume, storage: int) -> Volume:
        if isinstance(volume, Volume):
            return volume
        key = (id(volume.data), tuple(volume.data.shape), tuple(volume.voxel_size), tuple(volume.offset), storage)
        if key != self._key or self._data is not volume.data:
            if self._vol is not None:
                self._vol.release()
            self._vol = self.ctx.volume(volume, storage)
            self._key, self._data = key, volume.data
        return self._vol

    def release(self):
        if self._vol is not None:
            self._vol.release()
        self._vol, self._key, self._data = None, None, None


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


class LinearDynamicVolume:
    """LinearDynamicVolume(slope, offset) (img/lineardynamicvolume.h): voxels are
    slope * t + offset at time t (seconds); slope and offset are (Z, Y, X) float32
    arrays (or tensors) of one shape and voxel size."""

    def __init__(self, slope, offset, voxel_size: Sequence[float], volume_offset=(0.0, 0.0, 0.0)):
        if tuple(slope.shape) != tuple(offset.shape):
            raise ValueError("LinearDynamicVolume: offset and slope volumes have different sizes")
        self.slope = VoxelVolume(slope, voxel_size, volume_offset)
        self.offset = VoxelVolume(offset, voxel_size, volume_offset)

    def at(self, t: float) -> VoxelVolume:
        """The volume at time t, computed as the reference does (slope * float(t) + offset, FP32)."""
        s, o = np.asarray(self.slope.data, np.float32), np.asarray(self.offset.data, np.float32)
        return VoxelVolume((s * np.float32(t) + o).astype(np.float32), self.slope.voxel_size, self.slope.offset)


class DynamicProjectorExtension:
    """DynamicProjectorExtension (projectors/dynamicprojectorextension.cpp:37-60) around the
    B200 projector.  The reference re-projects every view with the volume set to that
    view's time.  For a LinearDynamicVolume the projection is linear in the voxels, so
    all views come from one batched projection of the slope and offset volumes and one
    combine launch; any other volume is projected as it is.  The volumes are uploaded on
    first use and stay resident while the same objects are projected again (they must
    not be modified in between); release() frees them."""

    def __init__(self, ctx: Context, settings: Optional[Settings] = None):
        self.ctx = ctx
        self.settings = settings or Settings()
        self._pm = None
        self._dims = None
        self._times = None
        self._resident = [_Resident(ctx), _Resident(ctx)]

    def configure(self, pmats, channels: int, rows: int, time_stamps: Sequence[float]) -> None:
        """pmats (views, modules, 3, 4) (host or device); time_stamps: one per view in
        seconds (AcquisitionSetup::View::timeStamp)."""
        if len(time_stamps) != int(pmats.shape[0]):
            raise ValueError("one time stamp per view")
        self._pm = pmats
        self._dims = (int(channels), int(rows))
        self._times = np.asarray(time_stamps, np.float64)

    def project(self, volume):
        import torch
        if self._pm is None:
            raise RuntimeError("DynamicProjectorExtension::project: configure() has not been called")
        C_, R = self._dims
        P = self._pm if hasattr(self._pm, "is_cuda") else torch.from_numpy(np.ascontiguousarray(self._pm)).cuda()
        if not isinstance(volume, LinearDynamicVolume):
            return self.ctx.project(self._resident[0].get(volume, self.settings.storage), P, C_, R, self.settings)
        vs = self._resident[0].get(volume.slope, self.settings.storage)
        vo = self._resident[1].get(volume.offset, self.settings.storage)
        V, M = int(P.shape[0]), int(P.shape[1])
        both = torch.empty((2, V, M, R, C_), dtype=torch.float32, device="cuda")
        self.ctx.project_batch([(vs, P, both[0]), (vo, P, both[1])], self.settings)
        out = self.ctx.combine_linear(both[0], both[1], self._times, torch.empty_like(both[0]))
        torch.cuda.synchronize()
        return out

    def release(self) -> None:
        """Free the resident volumes."""
        for r in self._resident:
            r.release()


class SpectralEffectsExtension:
    """SpectralEffectsExtension (projectors/spectraleffectsextension.cpp): the materials'
    density volumes projected in one batched launch, then every energy bin combined per
    pixel on the device.

    Linear case (:215-278; ctlcu_spectral_combine): the nested projector is linear.
    Around a nested PoissonNoiseExtension (the non-linear case, :285-314, :368-391;
    ctlcu_spectral_combine_noisy): the reference projects every material's attenuation
    volume per energy bin through projector | noise; here the density projections are
    scaled per bin (the projector is linear) and only the noise runs per (bin, material).

    The spectral inputs come from CTL's models, evaluated by the caller:
      mu_per_mm  [bins][materials]: meanMassAttenuationCoeff(E_b, binWidth) * 0.1 (cm -> mm)
      intensities [bins][views]:   RadiationEncoder bin intensities per view
      total_intensity [views]:     RadiationEncoder::totalIntensity()
      response [bins] or None:     the detector's spectral response model at E_b
      photons_per_pixel [bins][modules] or None: the nested PoissonNoiseExtension's i0 in
                                   each bin (photonsPerPixel with the bin's flux); None for
                                   the linear case
      fixed_seed:                  the nested noise extension's fixed seed (None: random)

    Material volumes given as VoxelVolumes are uploaded on first use and stay resident
    while the same objects are projected again (they must not be modified in between;
    pass resident Volumes to manage that explicitly); release() frees them."""

    def __init__(self, ctx: Context, settings: Optional[Settings] = None):
        self.ctx = ctx
        self.settings = settings or Settings()
        self._pm = None
        self._calls = 0
        self._resident = []

    def configure(self, pmats, channels: int, rows: int, mu_per_mm, intensities, total_intensity,
                  response=None, photons_per_pixel=None, fixed_seed: Optional[int] = None) -> None:
        self._pm = pmats
        self._dims = (int(channels), int(rows))
        self.mu = np.ascontiguousarray(mu_per_mm, np.float32)
        self.intensities = np.ascontiguousarray(intensities, np.float64)
        self.total = np.ascontiguousarray(total_intensity, np.float64)
        self.response = None if response is None else np.ascontiguousarray(response, np.float32)
        B, M = self.mu.shape
        V, Mod = int(pmats.shape[0]), int(pmats.shape[1])
        if self.intensities.shape != (B, V) or self.total.shape != (V,):
            raise ValueError("intensities must be [bins][views] and total_intensity [views]")
        if self.response is not None and self.response.shape != (B,):
            raise ValueError("response must hold one value per bin")
        self.i0 = None if photons_per_pixel is None else np.ascontiguousarray(photons_per_pixel, np.float32)
        if self.i0 is not None and self.i0.shape != (B, Mod):
            raise ValueError("photons_per_pixel must be [bins][modules]")
        self.fixed_seed = fixed_seed

    def is_linear(self) -> bool:
        return self.i0 is None

    def nested_calls(self) -> int:
        """Projections the reference makes through the nested chain per project():
        materials x bins not skipped (bins whose intensities sum to zero)."""
        live = int((np.abs(self.intensities.sum(axis=1)) > 1e-12).sum())
        return live * int(self.mu.shape[1])

    def project(self, material_densities: Sequence[VoxelVolume]):
        import torch
        if self._pm is None:
            raise RuntimeError("SpectralEffectsExtension::project: configure() has not been called")
        C_, R = self._dims
        M = len(material_densities)
        if M != self.mu.shape[1]:
            raise ValueError("one mass attenuation column per material")
        P = self._pm if hasattr(self._pm, "is_cuda") else torch.from_numpy(np.ascontiguousarray(self._pm)).cuda()
        V, Mod = int(P.shape[0]), int(P.shape[1])
        # the material volumes stay resident while the same objects are projected again
        if len(self._resident) != M:
            self.release()
            self._resident = [_Resident(self.ctx) for _ in range(M)]
        vols = [r.get(v, self.settings.storage) for r, v in zip(self._resident, material_densities)]
        try:
            projs = torch.empty((M, V, Mod, R, C_), dtype=torch.float32, device="cuda")
            self.ctx.project_batch([(vol, P, projs[m]) for m, vol in enumerate(vols)], self.settings)
            out = torch.empty((V, Mod, R, C_), dtype=torch.float32, device="cuda")
            from .projector import _ptr
            import ctypes as C
            stream = self.ctx._stream_for(0, out)
            resp = C.c_void_p(self.response.ctypes.data if self.response is not None else None)
            if self.i0 is None:
                self.ctx._check(self.ctx.lib.ctlcu_spectral_combine(
                    self.ctx.h, C.c_void_p(_ptr(projs)), M, V, Mod * R * C_, C.c_void_p(self.mu.ctypes.data),
                    C.c_void_p(self.intensities.ctypes.data), resp, int(self.mu.shape[0]),
                    C.c_void_p(self.total.ctypes.data), C.c_void_p(_ptr(out)), C.c_void_p(stream or None)))
                return out
            if self.fixed_seed is not None:
                seed = self.fixed_seed + self._calls  # the nested extension's next call
            else:
                seed = int.from_bytes(np.random.bytes(8), "little")
            self._calls += self.nested_calls()
            self.last_seed = seed
            self.ctx._check(self.ctx.lib.ctlcu_spectral_combine_noisy(
                self.ctx.h, C.c_void_p(_ptr(projs)), M, V, Mod, R * C_, C.c_void_p(self.mu.ctypes.data),
                C.c_void_p(self.intensities.ctypes.data), resp, int(self.mu.shape[0]),
                C.c_void_p(self.total.ctypes.data), C.c_void_p(self.i0.ctypes.data), C.c_uint64(seed % (1 << 64)),
                C.c_void_p(_ptr(out)), C.c_void_p(stream or None)))
            return out
        finally:
            torch.cuda.synchronize()

    def release(self) -> None:
        """Free the resident material volumes."""
        for r in getattr(self, "_resident", []):
            r.release()
        self._resident = []


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


def linear_saturation(lower_cap: float, upper_cap: float):
    """DetectorSaturationLinearModel(lowerCap, upperCap) (models/detectorsaturationmodels.cpp)."""
    from . import _lib as L
    return L.SaturationModel(L.SATURATION_LINEAR, float(lower_cap), float(upper_cap), 0.0, 0.0)


def spline_saturation(lower_cap: float, upper_cap: float, soft_lower: float, soft_upper: Optional[float] = None):
    """DetectorSaturationSplineModel(lowerCap, upperCap, softLower[, softUpper])."""
    from . import _lib as L
    su = soft_lower if soft_upper is None else soft_upper
    return L.SaturationModel(L.SATURATION_SPLINE, float(lower_cap), float(upper_cap), float(soft_lower), float(su))


class DetectorSaturationExtension:
    """DetectorSaturationExtension (projectors/detectorsaturationextension.cpp:96-226) around
    a B200 projector or extension: the nested projection, then the detector's saturation
    model applied on the device in its domain (ctlcu_detector_saturation).

      model:             linear_saturation(...) or spline_saturation(...)
      domain:            L.SATURATION_EXTINCTION, _PHOTON_COUNT or _INTENSITY
                         (AbstractDetector::saturationModelType())
      photons_per_pixel: [views][modules] or [modules]: SimpleCTSystem::photonsPerPixel()
                         after prepareView, for the photon count and intensity domains
      mean_energy:       [views] or scalar (keV): the centroid of each view's spectrum,
                         for the intensity domain (i0 = count x mean energy)"""

    def __init__(self, nested, model, domain: int, photons_per_pixel=None, mean_energy=None):
        from . import _lib as L
        if not isinstance(getattr(nested, "ctx", None), Context):
            raise TypeError("the nested projector must be a B200 projector or extension (with a Context)")
        if domain != L.SATURATION_EXTINCTION and photons_per_pixel is None:
            raise ValueError("the photon count and intensity domains need photons_per_pixel")
        if domain == L.SATURATION_INTENSITY and mean_energy is None:
            raise ValueError("the intensity domain needs the spectrum's mean energy")
        self.nested, self.ctx = nested, nested.ctx
        self.model, self.domain = model, int(domain)
        self.n0 = None if photons_per_pixel is None else np.asarray(photons_per_pixel, np.float32)
        self.mean_energy = None if mean_energy is None else np.asarray(mean_energy, np.float32)

    def is_linear(self) -> bool:
        return False

    def scale(self, n_views: int, n_modules: int):
        """The per-[view][module] count (or intensity) the extinctions refer to."""
        from . import _lib as L
        if self.domain == L.SATURATION_EXTINCTION:
            return None
        n0 = np.broadcast_to(self.n0, (n_views, n_modules)).astype(np.float32)
        if self.domain == L.SATURATION_INTENSITY:
            e = np.broadcast_to(self.mean_energy, (n_views,)).astype(np.float32)
            n0 = (n0 * e[:, None]).astype(np.float32)   # RadiationEncoder count x centroid, in float
        return n0

    def project(self, volume):
        out = self.nested.project(volume)
        V, M = int(out.shape[0]), int(out.shape[1])
        return self.ctx.detector_saturation(out, self.model, self.domain, self.scale(V, M))
