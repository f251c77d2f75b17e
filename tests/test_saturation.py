"""DetectorSaturationExtension (projectors/detectorsaturationextension.cpp:96-226) with
CTL's linear and spline saturation models (models/detectorsaturationmodels.cpp), on the
device, against the FP32 restatement in oracle.detector_saturation."""
import numpy as np
import pytest

import oracle

LINEAR, SPLINE = 0, 1


def test_linear_model_clamps():
    x = np.array([-5.0, 0.0, 0.5, 3.0, 7.9, 8.0, 100.0], np.float32)
    np.testing.assert_array_equal(oracle.saturation_value(x, LINEAR, 0.5, 8.0),
                                  np.array([0.5, 0.5, 0.5, 3.0, 7.9, 8.0, 8.0], np.float32))


@pytest.mark.parametrize("a,b,sa,sb", [(1.0, 10.0, 0.5, 1.0), (100.0, 5e4, 50.0, 2000.0), (0.0, 3.0, 0.25, 0.25)])
def test_spline_model_is_smooth_between_its_regimes(a, b, sa, sb):
    """Identity between a + sa and b - sb, the caps outside a - sa and b + sb, and
    value and slope continuous at the four joints (the reference's quadratic splines)."""
    f = lambda x: oracle.saturation_value(np.asarray(x, np.float32), SPLINE, a, b, sa, sb).astype(np.float64)
    lin = np.linspace(a + sa, b - sb, 50)
    np.testing.assert_allclose(f(lin), lin, rtol=1e-6)
    assert (f([a - sa - 1.0, a - 2 * sa]) == a).all() and (f([b + sb + 1.0, b + 2 * sb]) == b).all()
    for joint, left, right in ((a - sa, a, None), (a + sa, None, None), (b - sb, None, None), (b + sb, None, b)):
        h = 1e-3 * max(sa, sb)
        vl, vr = f(joint - h), f(joint + h)
        assert abs(vl - vr) <= 4 * h + 1e-5 * abs(joint)
    xs = np.linspace(a - 2 * sa, b + 2 * sb, 4001)
    assert (np.diff(f(xs)) >= -1e-6 * max(abs(a), abs(b), 1.0)).all()   # monotone non-decreasing


def test_count_domain_round_trip_without_saturation():
    """Caps far outside the data: the count domain returns the extinctions (up to FP32 exp/log)."""
    p = np.random.default_rng(0).uniform(0.0, 6.0, (3, 2, 4, 5)).astype(np.float32)
    n0 = np.array([[1e4, 2e4]] * 3, np.float32)
    out = oracle.detector_saturation(p, LINEAR, 0.0, 1e30, 0.0, 0.0, 1, n0)
    np.testing.assert_allclose(out, p, atol=2e-6)


def test_extension_scale_per_domain():
    """The [view][module] scale the extension hands to the device step: nothing in the
    extinction domain, the photon count, or count x the view's mean energy in FP32."""
    from ctl_b200 import _lib as L
    from ctl_b200.extensions import DetectorSaturationExtension, linear_saturation
    from ctl_b200.projector import Context

    class _Nested:
        ctx = Context.__new__(Context)   # type only: no device is touched here

    m = linear_saturation(0.0, 1.0)
    assert DetectorSaturationExtension(_Nested(), m, L.SATURATION_EXTINCTION).scale(3, 2) is None
    n0 = [1e4, 2e4]
    count = DetectorSaturationExtension(_Nested(), m, L.SATURATION_PHOTON_COUNT, photons_per_pixel=n0).scale(3, 2)
    np.testing.assert_array_equal(count, np.array([n0] * 3, np.float32))
    e = [50.0, 60.0, 70.0]
    inten = DetectorSaturationExtension(_Nested(), m, L.SATURATION_INTENSITY, photons_per_pixel=n0,
                                        mean_energy=e).scale(3, 2)
    np.testing.assert_array_equal(inten, (np.array([n0] * 3, np.float32) * np.float32(e)[:, None]))
    with pytest.raises(ValueError):
        DetectorSaturationExtension(_Nested(), m, L.SATURATION_PHOTON_COUNT)
    with pytest.raises(TypeError):
        DetectorSaturationExtension(object(), m, L.SATURATION_EXTINCTION)


# ---- device ----------------------------------------------------------------------------------

@pytest.fixture(scope="module")
def ctx():
    from ctl_b200.projector import Context
    c = Context(0)
    yield c
    c.close()


def _data(seed=1):
    rng = np.random.default_rng(seed)
    return rng.uniform(-0.5, 9.0, (4, 3, 16, 20)).astype(np.float32)


CASES = [
    # (kind, a, b, soft_a, soft_b, domain, scale): every regime of each model is populated
    (LINEAR, 0.5, 6.0, 0.0, 0.0, 0, None),
    (SPLINE, 0.5, 6.0, 0.4, 1.0, 0, None),
    (LINEAR, 50.0, 5000.0, 0.0, 0.0, 1, "count"),
    (SPLINE, 50.0, 5000.0, 30.0, 1500.0, 1, "count"),
    (SPLINE, 2e3, 2e5, 1e3, 5e4, 2, "intensity"),
]


def _scale(kind):
    n0 = np.array([[1e4, 2e4, 5e3]] * 4, np.float32) * np.array([1.0, 0.9, 1.1, 1.2], np.float32)[:, None]
    if kind == "count":
        return n0
    if kind == "intensity":
        return (n0 * np.array([55.0, 60.0, 62.5, 58.0], np.float32)[:, None]).astype(np.float32)
    return None


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("on_device", [False, True])
def test_device_saturation_matches_the_oracle(ctx, case, on_device):
    import torch
    from ctl_b200 import _lib as L
    kind, a, b, sa, sb, domain, sk = case
    p = _data()
    scale = _scale(sk)
    want = oracle.detector_saturation(p, kind, a, b, sa, sb, domain, scale)
    model = L.SaturationModel(kind, a, b, sa, sb)
    if on_device:
        d = torch.from_numpy(p.copy()).cuda()
        ctx.detector_saturation(d, model, domain, scale)
        ctx.sync()
        got = d.cpu().numpy()
    else:
        got = ctx.detector_saturation(p.copy(), model, domain, scale)
    if domain == 0:
        np.testing.assert_array_equal(got, want)   # the same FP32 operations, one rounding each
    else:
        finite = np.isfinite(want)
        assert (np.isfinite(got) == finite).all()
        np.testing.assert_allclose(got[finite], want[finite], rtol=2e-6, atol=2e-6)
    assert (got != p).mean() > 0.05   # the caps act on part of the data


class _Nested:
    """A nested B200 projector: the context projects the volume onto the scan (host result)."""

    def __init__(self, ctx, P, channels, rows):
        self.ctx, self.P, self.dims = ctx, P, (channels, rows)

    def project(self, vol):
        return self.ctx.project_volume(vol, self.P, *self.dims)


@pytest.mark.gpu
def test_saturation_extension_wraps_the_projector(ctx):
    from ctl_b200 import _lib as L
    from ctl_b200 import geometry as G
    from ctl_b200 import phantom as Ph
    from ctl_b200.extensions import DetectorSaturationExtension, spline_saturation
    from ctl_b200.projector import VoxelVolume
    vol = VoxelVolume(Ph.ellipsoid_phantom((32, 32, 24), (2.0, 2.0, 2.0), 5, seed=8) * 3.0, (2.0, 2.0, 2.0))
    P = G.circular_flat(4, 600.0, 900.0, G.FlatDetector(24, 20, 2.0, 2.0))
    nested = _Nested(ctx, P, 24, 20)
    plain = nested.project(vol)
    model = spline_saturation(200.0, 2e4, 100.0, 5e3)
    ext = DetectorSaturationExtension(nested, model, L.SATURATION_PHOTON_COUNT, photons_per_pixel=[3e4])
    assert not ext.is_linear()
    got = ext.project(vol)
    want = oracle.detector_saturation(plain, SPLINE, 200.0, 2e4, 100.0, 5e3, 1, np.full((4, 1), 3e4, np.float32))
    assert (want != plain).mean() > 0.05
    np.testing.assert_allclose(got, want, rtol=2e-6, atol=2e-6)
    with pytest.raises(ValueError):
        DetectorSaturationExtension(nested, model, L.SATURATION_INTENSITY, photons_per_pixel=[3e4])


@pytest.mark.gpu
def test_bad_saturation_arguments_are_refused(ctx):
    from ctl_b200 import _lib as L
    p = _data()
    for model, domain, scale in ((L.SaturationModel(LINEAR, 0.0, 1.0, 0.0, 0.0), 3, None),
                                 (L.SaturationModel(7, 0.0, 1.0, 0.0, 0.0), 0, None),
                                 (L.SaturationModel(SPLINE, 0.0, 1.0, 0.0, 0.1), 0, None),
                                 (L.SaturationModel(LINEAR, 0.0, 1.0, 0.0, 0.0), 1, None)):
        with pytest.raises(L.CtlcuError) as e:
            ctx.detector_saturation(p.copy(), model, domain, scale)
        assert e.value.status == L.ERR_INVALID_ARGUMENT
