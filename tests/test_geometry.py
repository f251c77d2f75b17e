"""Projection-matrix generation (CTL's GeometryEncoder for simple systems).

The oracle (oracle/geometry_oracle.py) is pinned to the reference's own golden
geometries, testing/testData/tubeGeo.den and cArmGeo.den, with the inputs and
the measure of testing/src/geometrytest.cpp:17-55, :122-139 (mean Frobenius
norm of the difference of normalised matrices < 1e-8).  The device encoder
(ctlcu_encode_geometry) is compared with the oracle for every protocol.
"""
import math

import numpy as np
import pytest

from oracle import geometry_oracle as GO
from tests._common import golden_geometry

GOLDEN_TOL = 1e-8   # geometrytest.cpp:124
# device vs oracle, the same absolute measure: FP64 on both sides, only the
# rounding of sin/cos/sqrt differs (entries reach 2.4e5, so 1e-9 is ~1e-15 relative)
DEVICE_TOL = 1e-9


def test_oracle_reproduces_the_reference_golden_geometries():
    g = golden_geometry()
    for name, make in (("tube", GO.golden_tube_setup), ("carm", GO.golden_carm_setup)):
        det, traj, n = make()
        P = GO.encode_full_geometry(det, traj, n)
        assert P.shape == g[name + "_pmats"].shape
        assert GO.pmat_difference(P, g[name + "_pmats"]) < GOLDEN_TOL, name


def test_oracle_source_positions_match_the_reference_decomposition():
    """The source recovered from each encoded matrix (the reference's own
    determineSource output, stored with the golden vectors) is the gantry's."""
    g = golden_geometry()
    det, traj, n = GO.golden_carm_setup()
    for v in range(n):
        src = GO.gantry_state(traj, v, n, det)[0]
        np.testing.assert_allclose(src, g["carm_src"][v], rtol=0, atol=1e-9)


def _cases():
    deg = math.radians
    cyl = GO.Detector(16, 64, 1.0, 1.0, modules=40, angulation=deg(1.0), spacing=0.2)
    cyl_skew = GO.Detector(24, 8, 0.8, 1.1, modules=7, angulation=deg(2.5), spacing=0.5, skew=0.01)
    flat = GO.Detector(512, 384, 0.6, 0.7, flat_panel=True)
    return {
        "tube_helical": (cyl, GO.Trajectory("helical", sdd=1000.0, sid=550.0, pitch=deg(90.0),
                                            angle_increment=deg(3.6), pitch_increment=1.0), 10),
        "carm_wobble": (cyl, GO.Trajectory("wobble", carm_span=1200.0, source_to_iso=750.0,
                                           angle_span=deg(200.0), wobble_angle=deg(20.0), wobble_freq=5.0), 30),
        "tilted_helical_start": (cyl_skew, GO.Trajectory("helical", sdd=1040.0, sid=570.0, tilt=deg(7.0),
                                                         angle_increment=deg(1.0), pitch_increment=0.7,
                                                         start_pitch=-20.0, start_angle=deg(33.0)), 50),
        "axial": (cyl, GO.Trajectory("axial", sdd=1000.0, sid=600.0, pitch=12.5, start_angle=deg(10.0)), 37),
        "short_scan_flat_default_span": (flat, GO.Trajectory("short_scan", carm_span=1200.0,
                                                             source_to_iso=750.0, angle_span=-deg(1.0)), 45),
        "short_scan_cyl_span": (cyl, GO.Trajectory("short_scan", carm_span=1100.0, source_to_iso=700.0,
                                                   angle_span=deg(210.0), start_angle=deg(-15.0)), 21),
        "short_scan_cyl_default_span": (cyl, GO.Trajectory("short_scan", carm_span=1100.0,
                                                           source_to_iso=700.0, angle_span=-1.0), 21),
        "circle_plus_line": (flat, GO.Trajectory("circle_plus_line", carm_span=1200.0, source_to_iso=750.0,
                                                 angle_span=deg(220.0), line_length=180.0, line_fraction=0.3), 40),
        "single_view": (flat, GO.Trajectory("wobble", carm_span=1200.0, source_to_iso=750.0,
                                            angle_span=deg(90.0), wobble_angle=deg(5.0), wobble_freq=1.0), 1),
    }


def test_oracle_matrices_are_normalised_with_positive_determinant():
    for name, (det, traj, n) in _cases().items():
        P = GO.encode_full_geometry(det, traj, n)
        M = P[..., :3]
        np.testing.assert_allclose(np.linalg.norm(M[..., 2, :], axis=-1), 1.0, rtol=1e-12, err_msg=name)
        assert (np.linalg.det(M) > 0).all(), name


def _to_device_desc(det, traj):
    from ctl_b200 import encoder as E
    if det.flat_panel:
        d = E.FlatPanelDetector((det.channels, det.rows), (det.pixel_w, det.pixel_h), det.skew)
    else:
        d = E.CylindricalDetector((det.channels, det.rows), (det.pixel_w, det.pixel_h), det.modules,
                                  det.angulation, det.spacing, det.skew)
    if traj.kind in ("helical", "axial"):
        g = E.TubularGantry(traj.sdd, traj.sid, 0.0, traj.pitch, traj.tilt)
        p = (E.HelicalTrajectory(traj.angle_increment, traj.pitch_increment, traj.start_pitch, traj.start_angle)
             if traj.kind == "helical" else E.AxialScanTrajectory(traj.start_angle))
    else:
        g = E.CarmGantry(traj.carm_span)
        if traj.kind == "wobble":
            p = E.WobbleTrajectory(traj.angle_span, traj.source_to_iso, traj.start_angle, traj.wobble_angle,
                                   traj.wobble_freq)
        elif traj.kind == "short_scan":
            p = E.ShortScanTrajectory(traj.source_to_iso, traj.start_angle, traj.angle_span)
        else:
            p = E.CirclePlusLineTrajectory(traj.angle_span, traj.source_to_iso, traj.line_length,
                                           traj.line_fraction, traj.start_angle)
    return d, g, p


@pytest.fixture(scope="module")
def ctx():
    from ctl_b200.projector import Context
    c = Context(0)
    yield c
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(_cases()))
def test_device_encoder_matches_the_oracle(ctx, name):
    from ctl_b200 import encoder as E
    det, traj, n = _cases()[name]
    d, g, p = _to_device_desc(det, traj)
    setup = E.AcquisitionSetup(d, g, n)
    setup.apply_preparation_protocol(p)
    got = E.GeometryEncoder.encode_full_geometry(setup, ctx)
    want = GO.encode_full_geometry(det, traj, n)
    assert got.shape == want.shape
    assert GO.pmat_difference(got, want) < DEVICE_TOL, name
    assert np.abs(got - want).max() / np.abs(want).max() < 1e-12, name


@pytest.mark.gpu
def test_device_encoder_reproduces_the_golden_geometries_into_device_memory(ctx):
    import torch
    from ctl_b200 import encoder as E
    g = golden_geometry()
    for name, make in (("tube", GO.golden_tube_setup), ("carm", GO.golden_carm_setup)):
        det, traj, n = make()
        d, gan, p = _to_device_desc(det, traj)
        setup = E.AcquisitionSetup(d, gan, n)
        setup.apply_preparation_protocol(p)
        out = torch.empty((n, 40, 3, 4), dtype=torch.float64, device="cuda")
        E.GeometryEncoder.encode_full_geometry(setup, ctx, out=out)
        assert GO.pmat_difference(out.cpu().numpy(), g[name + "_pmats"]) < GOLDEN_TOL, name


@pytest.mark.gpu
def test_device_encoder_rejects_bad_systems(ctx):
    from ctl_b200 import _lib as L
    from ctl_b200 import encoder as E
    bad = [
        (E.CylindricalDetector((0, 8), (1, 1), 4, 0.01, 0.0), E.TubularGantry(1000, 500), E.AxialScanTrajectory()),
        (E.CylindricalDetector((8, 8), (1, 1), 4, 0.0, 0.0), E.TubularGantry(1000, 500), E.AxialScanTrajectory()),
        (E.FlatPanelDetector((8, 8), (1, 1)), E.CarmGantry(0.0), E.ShortScanTrajectory(700.0)),
        (E.FlatPanelDetector((8, 8), (1, 1)), E.TubularGantry(-1.0, 500), E.AxialScanTrajectory()),
    ]
    for d, g, p in bad:
        s = E.AcquisitionSetup(d, g, 4)
        s.apply_preparation_protocol(p)
        with pytest.raises(L.CtlcuError) as e:
            E.GeometryEncoder.encode_full_geometry(s, ctx)
        assert e.value.status == L.ERR_INVALID_ARGUMENT
    with pytest.raises(ValueError):
        E.AcquisitionSetup(E.FlatPanelDetector((8, 8), (1, 1)), E.CarmGantry(1000.0), 4) \
            .apply_preparation_protocol(E.HelicalTrajectory(0.1))
