"""The FP64 oracle, pinned before it is trusted.

Pins, in order:
  * setup math: packed QR and source position equal the reference's own
    mat::QRdecomposition / ProjectionMatrix::sourcePosition output on CTL's
    golden geometries (tests/golden/geometry.npz from testing/testData/*.den);
  * the source-position known answer of projectionmatrixtest.cpp:8-13,49-52;
  * projections equal the reference's own ray_caster kernels (compiled for
    the CPU, tests/golden/projections.npz) within the FP32-vs-FP64 gap;
  * closed-form answers: uniform cube chord length, a ray that misses, a
    single hot voxel.
"""
import math

import numpy as np
import pytest

import oracle
from ctl_b200 import geometry as G
from tests._common import golden_cases, golden_geometry, rel_err


@pytest.fixture(scope="module", autouse=True)
def _built():
    oracle.build(with_ref=False)


def test_setup_matches_reference_mat_code():
    g = golden_geometry()
    for key in ("tube", "carm"):
        qr, src = oracle.view_setup(g[f"{key}_pmats"], "fp64")
        np.testing.assert_allclose(qr, g[f"{key}_qr"], rtol=0, atol=1e-9 * np.abs(g[f"{key}_qr"]).max())
        np.testing.assert_allclose(src, g[f"{key}_src"], rtol=0, atol=1e-9)


def test_golden_geometry_sources():
    """tubeGeo: SID 550 helical; cArmGeo: SID 750 wobble (geometrytest.cpp:21-56)."""
    g = golden_geometry()
    assert g["tube_pmats"].shape == (10, 40, 3, 4)
    assert g["carm_pmats"].shape == (30, 40, 3, 4)
    np.testing.assert_allclose(np.linalg.norm(g["tube_src"][:, :2], axis=1), 550.0, atol=1e-9)
    np.testing.assert_allclose(np.linalg.norm(g["carm_src"][0]), 750.0, atol=1e-9)
    # every module of a view shares the source (raycasterprojector.cpp:324-325)
    P = g["tube_pmats"]
    for v in range(P.shape[0]):
        for m in (0, 17, 39):
            _, s = oracle.view_setup(P[v:v + 1, m:m + 1], "fp64")
            np.testing.assert_allclose(s[0], g["tube_src"][v], atol=1e-8)


def test_source_position_known_answer():
    """P = -compose(K, rotX(-90 deg), C=(0,300,0)) / 300 has its source at C."""
    K = np.array([[1000.0, 0, 300], [0, 1000.0, 250], [0, 0, 1]])
    a = math.radians(-90.0)
    R = np.array([[1, 0, 0], [0, math.cos(a), -math.sin(a)], [0, math.sin(a), math.cos(a)]])
    P = -G.compose(K, R, np.array([0.0, 300.0, 0.0])) / 300.0
    _, src = oracle.view_setup(P[None, None], "fp64")
    assert np.linalg.norm(src[0] - np.array([0.0, 300.0, 0.0])) <= 1e-12 * 300


def test_decompose_sign_rule():
    """det M < 0 negates R so that R^-1 Q^T [x,y,1] still points at the detector."""
    K = np.array([[1000.0, 0, 300], [0, 1000.0, 250], [0, 0, 1]])
    P = G.compose(K, np.eye(3), np.array([0.0, 0.0, -500.0]))
    for scale in (1.0, -1.0 / 300.0):
        qr, _ = oracle.view_setup((scale * P)[None, None], "fp64")
        q = qr[0, 0]
        Q = q[:9].reshape(3, 3)
        R = np.array([[q[9], q[10], q[11]], [0, q[12], q[13]], [0, 0, q[14]]])
        d = np.linalg.solve(R, Q.T @ np.array([300.0, 250.0, 1.0]))
        assert np.linalg.det(R) > 0
        assert d[2] > 0 and abs(d[0]) < 1e-12 * abs(d[2]) and abs(d[1]) < 1e-12 * abs(d[2])


@pytest.mark.parametrize("case", golden_cases(), ids=lambda c: c[0]["name"])
def test_oracle_matches_reference_kernel(case):
    m, vol, P, ref = case
    out, _ = oracle.project_fp64(vol, m["voxel"], P, m["channels"], m["rows"], offset_mm=m["offset"],
                                 rays=m["rays"], ray_sampling=m["ray_sampling"], upsampling=m["upsampling"],
                                 interpolate=m["interpolate"])
    e = rel_err(ref, out)
    if m["upsampling"] == 0 and m["interpolate"]:
        # the reference sums the mean voxel in FP32 (raycasterprojector.cpp:603-606)
        assert e.max() < 3e-4
    elif m["interpolate"]:
        # FP32 positions/weights in the reference vs FP64 here
        assert e.max() < 5e-4 and e.mean() < 1e-5
    else:
        # nearest voxel: an FP32 position may pick the neighbouring voxel
        assert np.quantile(e, 0.999) < 1e-3 and e.mean() < 1e-4


def _center_view(n_det=33, sid=750.0, sdd=1000.0, pitch=0.5):
    det = G.FlatDetector(n_det, n_det, pitch, pitch)
    return G.circular_flat(1, sid, sdd, det)


def test_uniform_cube_chord():
    """Central ray along x through a uniform cube: line integral = mu * edge."""
    n, v, mu = 20, 2.0, 0.02
    vol = np.full((n, n, n), mu, np.float32)
    P = _center_view()
    out, _ = oracle.project_fp64(vol, (v, v, v), P, 33, 33)
    inc = 0.3 * v
    assert abs(out[0, 0, 16, 16] - mu * n * v) <= 2 * mu * inc


def test_miss_is_zero():
    n, v = 8, 1.0
    vol = np.ones((n, n, n), np.float32)
    det = G.FlatDetector(400, 400, 1.0, 1.0)
    P = G.circular_flat(1, 750.0, 1000.0, det)
    out, _ = oracle.project_fp64(vol, (v, v, v), P, 400, 400)
    assert out[0, 0, 0, 0] == 0.0 and out[0, 0, 399, 399] == 0.0
    assert out[0, 0, 200, 200] > 0.0


def test_hot_voxel_tent():
    """One voxel of value 1: the trilinear tent integrates to one voxel length."""
    n, v = 5, 1.0
    vol = np.zeros((n, n, n), np.float32)
    vol[2, 2, 2] = 1.0
    P = _center_view(n_det=33, pitch=0.1)
    out, _ = oracle.project_fp64(vol, (v, v, v), P, 33, 33)
    assert abs(out[0, 0, 16, 16] - v) <= 0.3 * v * 1.0


def test_nearest_box_without_padding():
    """No interpolation: the box is not padded (raycasterprojector_no_interp.cl:97-98)."""
    n, v, mu = 16, 1.0, 0.05
    vol = np.full((n, n, n), mu, np.float32)
    P = _center_view()
    out, _ = oracle.project_fp64(vol, (v, v, v), P, 33, 33, interpolate=False)
    assert abs(out[0, 0, 16, 16] - mu * n * v) <= 2 * mu * 0.3 * v


def test_upsampling_replication_equals_physical():
    """Virtual f=2 equals projecting the 2x-replicated volume with half voxels."""
    rng = np.random.default_rng(0)
    vol = rng.uniform(0, 0.05, (6, 7, 8)).astype(np.float32)
    big = vol.repeat(2, 0).repeat(2, 1).repeat(2, 2)
    det = G.FlatDetector(24, 20, 1.0, 1.0)
    P = G.circular_flat(3, 750.0, 1000.0, det)
    a, _ = oracle.project_fp64(vol, (2.0, 2.0, 2.0), P, 24, 20, upsampling=2)
    b, _ = oracle.project_fp64(big, (1.0, 1.0, 1.0), P, 24, 20, upsampling=1)
    np.testing.assert_array_equal(a, b)


def test_sample_count_formula():
    """S = sum over rays of floor(tmax) + 2 - floor(tmin); misses add nothing."""
    n, v = 10, 1.0
    vol = np.ones((n, n, n), np.float32)
    P = _center_view(n_det=33)
    _, S1 = oracle.project_fp64(vol, (v, v, v), P, 33, 33)
    _, S2 = oracle.project_fp64(vol, (v, v, v), P, 33, 33, rays=(2, 2))
    assert S1 > 0 and 3.9 * S1 < S2 < 4.1 * S1


@pytest.mark.skipif(not oracle.ref_available(), reason="reference kernel not built here")
def test_oracle_matches_live_reference_on_config1_slice():
    """A slice of the 64^3 -> 128^2 circular configuration, against the reference kernel run live."""
    from ctl_b200 import phantom
    vol = phantom.ellipsoid_phantom((64, 64, 64), (2, 2, 2), 10, seed=1)
    P = G.circular_flat(90, 750.0, 1000.0, G.FlatDetector(128, 128, 1.0, 1.0))[::15]
    a, _ = oracle.project_fp64(vol, (2, 2, 2), P, 128, 128)
    b = oracle.project_ref(vol, (2, 2, 2), P, 128, 128)
    e = rel_err(b, a)
    assert e.max() < 1e-4 and e.mean() < 1e-6
