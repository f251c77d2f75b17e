"""Host-side logic that needs no GPU: settings, parameters, geometry, DEN files."""
import math
import os

import numpy as np
import pytest

from ctl_b200 import _lib as L
from ctl_b200 import geometry as G
from ctl_b200.den import read_den, read_full_geometry, write_den
from ctl_b200.projector import CudaRayCasterProjector, ProjectionData, Settings, ViewDimensions


def test_optimized_for_square_pixels_and_large_voxels():
    """optimizedFor (raycasterprojector.cpp:482-521): 2 mm voxels, 1 mm pixels -> f = 2."""
    s = Settings.optimized_for(2.0, (1.0, 1.0))
    assert s.rays_per_pixel == [1, 1] and s.volume_upsampling == 2


def test_optimized_for_small_voxels_adds_rays():
    s = Settings.optimized_for(0.5, (1.0, 1.0))
    assert s.rays_per_pixel == [2, 2] and s.volume_upsampling == 1


def test_optimized_for_rectangular_pixels():
    s = Settings.optimized_for(1.0, (1.0, 2.0))
    assert s.rays_per_pixel == [1, 2]
    s = Settings.optimized_for(1.0, (3.0, 1.0))
    assert s.rays_per_pixel == [3, 1]


def test_optimized_for_singular_pixels():
    with pytest.raises(RuntimeError):
        Settings.optimized_for(1.0, (0.0, 1.0))


def _bare_projector():
    # parameter logic only: no device needed
    p = CudaRayCasterProjector.__new__(CudaRayCasterProjector)
    p._settings = Settings()
    p._geometry = None
    p.notifier = []
    return p


def test_parameter_keys_round_trip():
    """The reference's keys (raycasterprojector.cpp:69-91) plus the B200 options."""
    p = _bare_projector()
    par = p.parameter()
    for k in ("Rays per pixel X", "Rays per pixel Y", "Ray sampling step length",
              "Volume upsampling factor", "Interpolate"):
        assert k in par
    par.update({"Rays per pixel X": 3, "Ray sampling step length": 0.5, "Interpolate": False,
                "Accumulation": "kahan", "Storage": "bf16", "Interpolation mode": "texture"})
    p.set_parameter(par)
    s = p.settings()
    assert s.rays_per_pixel == [3, 1] and abs(s.ray_sampling - 0.5) < 1e-12 and not s.interpolate
    assert s.accum == L.ACCUM_KAHAN and s.storage == L.BF16 and s.interp_mode == L.INTERP_TEXTURE
    v = p.to_variant()
    assert v["#"] == "CudaRayCasterProjector" and v["parameters"]["Rays per pixel X"] == 3
    q = _bare_projector()
    q.from_variant(v)
    assert q.parameter() == p.parameter()


def test_set_parameter_defaults():
    p = _bare_projector()
    p.set_parameter({})
    s = p.settings()
    assert s.rays_per_pixel == [1, 1] and abs(s.ray_sampling - 0.3) < 1e-7
    assert s.volume_upsampling == 1 and s.interpolate


def test_project_before_configure_raises():
    p = _bare_projector()
    with pytest.raises(RuntimeError):
        p.project(None)


def test_projection_data_composite_sum():
    vd = ViewDimensions(4, 3, 2)
    a = ProjectionData(vd, np.ones((5, 2, 3, 4), np.float32))
    b = ProjectionData(vd, 2 * np.ones((5, 2, 3, 4), np.float32))
    a += b
    assert a.nb_views() == 5 and np.all(a.numpy() == 3)


def test_generated_pmats_are_normalised():
    det = G.FlatDetector(64, 48, 0.6, 0.6)
    P = G.circular_flat(12, 750.0, 1200.0, det, angle_range=math.radians(214.6),
                        rng=np.random.default_rng(1), jitter_mm=0.5, tilt_deg=0.2)
    for v in range(P.shape[0]):
        M = P[v, 0, :, :3]
        assert abs(np.linalg.norm(M[2]) - 1.0) < 1e-12 and np.linalg.det(M) > 0
        C = -np.linalg.solve(M, P[v, 0, :, 3])
        assert abs(np.linalg.norm(C[:2]) - 750.0) < 1.5


def test_generated_pmats_project_isocentre_to_detector_centre():
    det = G.FlatDetector(65, 33, 1.0, 1.0)
    P = G.circular_flat(8, 750.0, 1000.0, det)
    for v in range(8):
        x = P[v, 0] @ np.array([0.0, 0.0, 0.0, 1.0])
        np.testing.assert_allclose(x[:2] / x[2], [32.0, 16.0], atol=1e-9)


def test_helical_modules_share_the_source():
    P = G.helical_cylindrical(4, 1.0, 570.0, 1040.0, 8, 16, 16, 1.0, -10.0, 10.0)
    for v in range(4):
        srcs = [-np.linalg.solve(P[v, m, :, :3], P[v, m, :, 3]) for m in range(8)]
        np.testing.assert_allclose(srcs, np.repeat(srcs[:1], 8, 0), atol=1e-9)


def test_den_round_trip(tmp_path):
    a = np.arange(2 * 3 * 4, dtype=np.float64).reshape(2, 3, 4)
    f = os.path.join(tmp_path, "x.den")
    write_den(f, a)
    np.testing.assert_array_equal(read_den(f, np.float64), a)
    g = read_full_geometry(f, 1)
    assert g.shape == (2, 1, 3, 4)
