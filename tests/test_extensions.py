"""Extension chains as batched device work: ArealFocalSpotExtension (and Poisson
noise on its result), against the oracle and with the reference's own
statistical test strategy (testing/src/projectortest.cpp:149-234).
"""
import math

import numpy as np
import pytest

import oracle
from oracle import geometry_oracle as GO
from tests._common import rel_err

TOL = 1e-4


def test_discretization_grid_matches_the_oracle_restatement():
    from ctl_b200.extensions import discretization_grid
    for nx, ny in ((1, 1), (2, 2), (3, 1), (1, 4), (3, 5)):
        assert discretization_grid(nx, ny) == GO.focal_spot_grid(nx, ny)
    assert discretization_grid(2, 2) == [(-0.5, -0.5), (-0.5, 0.5), (0.5, -0.5), (0.5, 0.5)]


def test_resident_volume_is_uploaded_once_per_array():
    """The extensions' volume cache: one upload while the same array is projected again,
    a new upload (and the old one released) for another array, voxel size or storage."""
    from ctl_b200.extensions import _Resident
    from ctl_b200.projector import VoxelVolume

    class _Vol:
        released = False

        def release(self):
            self.released = True

    class _Ctx:
        uploads = 0

        def volume(self, vol, storage):
            self.uploads += 1
            return _Vol()

    ctx = _Ctx()
    cache = _Resident(ctx)
    a = np.zeros((4, 5, 6), np.float32)
    first = cache.get(VoxelVolume(a, (1.0, 1.0, 1.0)), 0)
    assert cache.get(VoxelVolume(a, (1.0, 1.0, 1.0)), 0) is first and ctx.uploads == 1
    b = np.zeros((4, 5, 6), np.float32)
    second = cache.get(VoxelVolume(b, (1.0, 1.0, 1.0)), 0)
    assert ctx.uploads == 2 and first.released and second is not first
    cache.get(VoxelVolume(b, (2.0, 1.0, 1.0)), 0)
    cache.get(VoxelVolume(b, (2.0, 1.0, 1.0)), 1)
    assert ctx.uploads == 4
    cache.release()
    assert cache.get(VoxelVolume(b, (2.0, 1.0, 1.0)), 1) is not None and ctx.uploads == 5


def test_oracle_source_shift_moves_the_decomposed_source():
    """The source that the reference's decomposition recovers from a shifted
    matrix is the gantry's source moved by sourceRotation * shift."""
    det = GO.Detector(64, 48, 2.0, 2.0, flat_panel=True)
    traj = GO.Trajectory("short_scan", carm_span=1200.0, source_to_iso=750.0, angle_span=math.radians(90.0))
    shift = np.array([2.5, -1.5, 0.0])
    P = GO.encode_full_geometry(det, traj, 5, source_shift=shift)
    _, src = oracle.view_setup(P)
    for v in range(5):
        s0, _, _, R = GO.gantry_state(traj, v, 5, det)
        np.testing.assert_allclose(src[v], s0 + R @ shift, atol=1e-9)


# ---- device ----------------------------------------------------------------------------------

def _system():
    """A 64 x 48 flat panel of 2 mm pixels on a C-arm (SID 750, span 1200), as in the
    reference's Poisson/focal-spot test, over a short arc."""
    from ctl_b200 import encoder as E
    det = GO.Detector(64, 48, 2.0, 2.0, flat_panel=True)
    traj = GO.Trajectory("short_scan", carm_span=1200.0, source_to_iso=750.0, angle_span=math.radians(60.0),
                         start_angle=math.radians(10.0))
    setup = E.AcquisitionSetup(E.FlatPanelDetector((64, 48), (2.0, 2.0)), E.CarmGantry(1200.0), 4)
    setup.apply_preparation_protocol(E.ShortScanTrajectory(750.0, math.radians(10.0), math.radians(60.0)))
    return det, traj, setup


def _volume():
    from ctl_b200 import phantom as Ph
    return Ph.ellipsoid_phantom((48, 48, 40), (2.0, 2.0, 2.0), 8, seed=21)


def _oracle_focal_spot(vol, det, traj, n_views, spot, grid, low):
    subs = []
    for x, y in GO.focal_spot_grid(*grid):
        P = GO.encode_full_geometry(det, traj, n_views, source_shift=(x * spot[0], y * spot[1], 0.0))
        p, _ = oracle.project_fp64(vol, (2.0, 2.0, 2.0), P, det.channels, det.rows)
        subs.append(p.astype(np.float64))
    subs = np.stack(subs)
    return subs.mean(0) if low else -np.log(np.exp(-subs).mean(0))


@pytest.fixture(scope="module")
def ctx():
    from ctl_b200.projector import Context
    c = Context(0)
    yield c
    c.close()


@pytest.mark.gpu
def test_shifted_device_encoder_matches_the_oracle(ctx):
    from ctl_b200 import encoder as E
    det, traj, setup = _system()
    shifts = np.array([[-2.5, -2.5, 0], [-2.5, 2.5, 0], [2.5, -2.5, 0], [2.5, 2.5, 0.0]])
    got = E.GeometryEncoder.encode_full_geometry(setup, ctx, source_shifts=shifts)
    assert got.shape == (16, 1, 3, 4)
    for k, s in enumerate(shifts):
        want = GO.encode_full_geometry(det, traj, 4, source_shift=s)
        assert GO.pmat_difference(got[4 * k: 4 * k + 4], want) < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("grid,low", [((2, 2), False), ((3, 2), False), ((2, 2), True), ((1, 1), False)])
def test_focal_spot_extension_matches_the_oracle(ctx, grid, low):
    from ctl_b200.extensions import ArealFocalSpotExtension
    from ctl_b200.projector import VoxelVolume
    det, traj, setup = _system()
    vol = _volume()
    ext = ArealFocalSpotExtension(ctx, discretization=grid, low_extinction_approximation=low)
    ext.configure(setup, (5.0, 5.0))
    got = ext.project(VoxelVolume(vol, (2.0, 2.0, 2.0))).cpu().numpy()
    want = _oracle_focal_spot(vol, det, traj, 4, (5.0, 5.0), grid, low)
    assert rel_err(got, want).max() <= TOL
    ext.release()


@pytest.mark.gpu
def test_focal_spot_and_noise_follow_the_reference_test_strategy(ctx):
    """projectortest.cpp:149-234: the same pose repeated, Poisson noise on the
    focal-spot projections; the repetition mean of the counts matches the clean
    counts to 1% and the mean equals the variance (Poisson)."""
    from ctl_b200 import encoder as E
    from ctl_b200.extensions import ArealFocalSpotExtension, PoissonNoiseExtension
    from ctl_b200.projector import VoxelVolume
    reps, i0 = 400, 5000.0
    setup = E.AcquisitionSetup(E.FlatPanelDetector((50, 50), (2.0, 2.0)), E.CarmGantry(1200.0), reps)
    setup.apply_preparation_protocol(E.ShortScanTrajectory(750.0, math.radians(30.0), 0.0))  # one pose, repeated
    vol = VoxelVolume(_volume(), (2.0, 2.0, 2.0))
    clean_ext = ArealFocalSpotExtension(ctx, discretization=(2, 2))
    clean_ext.configure(setup, (5.0, 5.0))
    clean = clean_ext.project(vol).cpu().numpy()[0, 0].astype(np.float64)
    noisy_ext = PoissonNoiseExtension(clean_ext, i0, fixed_seed=11)
    noisy = noisy_ext.project(vol).cpu().numpy()[:, 0].astype(np.float64)
    counts = i0 * np.exp(-noisy)
    clean_counts = i0 * np.exp(-clean)
    mean, var = counts.mean(0), counts.var(0, ddof=1)
    assert abs(mean.mean() / clean_counts.mean() - 1.0) < 0.01
    diff = (mean - var) / mean
    assert abs(diff.mean()) < 0.05 and diff.std() < 0.25
    clean_ext.release()


# ---- spectral effects -----------------------------------------------------------------------

@pytest.mark.gpu
def test_spectral_extension_matches_the_oracle(ctx):
    """Two material densities, four energy bins (one with zero intensity, which the
    reference skips), per-view intensities and a detector response: one batched
    projection of the materials and the device combine, against per-material oracle
    projections combined in FP64 (spectraleffectsextension.cpp:215-278, :333-353)."""
    from ctl_b200 import geometry as G
    from ctl_b200 import phantom as Ph
    from ctl_b200.extensions import SpectralEffectsExtension
    from ctl_b200.projector import VoxelVolume
    vox = (2.0, 2.0, 2.0)
    water = Ph.ellipsoid_phantom((40, 40, 32), vox, 5, seed=41) * 40.0   # densities, g/cm^3
    bone = Ph.ellipsoid_phantom((40, 40, 32), vox, 3, seed=42) * 20.0
    P = G.circular_flat(5, 750.0, 1000.0, G.FlatDetector(48, 40, 2.0, 2.0))
    mu = np.array([[0.0268, 0.0573], [0.0206, 0.0303], [0.0, 0.0], [0.0184, 0.0223]], np.float32)  # 1/mm per g/cm^3
    rng = np.random.default_rng(5)
    inten = rng.uniform(100.0, 1000.0, (4, 5))
    inten[2] = 0.0                          # an empty bin
    response = np.array([0.9, 0.95, 1.0, 0.8], np.float32)
    total = inten.sum(0)
    ext = SpectralEffectsExtension(ctx)
    ext.configure(P, 48, 40, mu, inten, total, response)
    got = ext.project([VoxelVolume(water, vox), VoxelVolume(bone, vox)]).cpu().numpy()
    pw, _ = oracle.project_fp64(water, vox, P, 48, 40)
    pb, _ = oracle.project_fp64(bone, vox, P, 48, 40)
    acc = np.zeros(pw.shape)
    for b in (0, 1, 3):
        e = pw.astype(np.float64) * mu[b, 0] + pb.astype(np.float64) * mu[b, 1]
        acc += inten[b][:, None, None, None] * np.exp(-e) * response[b]
    want = np.log(total[:, None, None, None] / acc)
    assert rel_err(got, want).max() <= TOL


def _noisy_spectral_composition(projs, mu, inten, response, total, i0, seed):
    """The reference's non-linear loop (spectraleffectsextension.cpp:285-314, :368-391) on the
    CPU: per bin not skipped, each material's projection mu[b][m] * proj_m through the noise
    step (oracle.poisson_noise, the device algorithm restated; seed + c for the c-th nested
    call), summed over materials, to intensity, detector response, summed over bins, to
    extinction.  FP32 like the device."""
    M = projs.shape[0]
    acc = np.zeros(projs.shape[1:], np.float32)
    call = 0
    for b in range(mu.shape[0]):
        if abs(inten[b].sum()) <= 1e-12:
            continue
        e = np.zeros(projs.shape[1:], np.float32)
        for m in range(M):
            em = (projs[m] * np.float32(mu[b, m])).astype(np.float32)
            if abs(float(i0[b].sum())) <= 1e-12:
                e += em
            else:
                noisy, _ = oracle.poisson_noise(em, i0[b], seed + call)
                e += noisy
            call += 1
        acc += (inten[b].astype(np.float32)[:, None, None, None] * np.exp(-e) * np.float32(response[b]))
    return np.log(total.astype(np.float32)[:, None, None, None] / acc), call


def test_spectral_configure_checks_its_inputs_and_counts_nested_calls():
    """configure() rejects inputs of the wrong shapes; the nested projections per call are
    materials x bins with intensity (a bin without intensity makes no call)."""
    from ctl_b200.extensions import SpectralEffectsExtension
    from ctl_b200.projector import Context
    ext = SpectralEffectsExtension(Context.__new__(Context))   # type only: no device is touched
    P = np.zeros((5, 2, 3, 4))
    mu = np.ones((4, 3), np.float32)
    inten = np.ones((4, 5))
    inten[1] = 0.0
    ext.configure(P, 8, 6, mu, inten, inten.sum(0))
    assert ext.is_linear() and ext.nested_calls() == 3 * 3
    ext.configure(P, 8, 6, mu, inten, inten.sum(0), photons_per_pixel=np.ones((4, 2)), fixed_seed=1)
    assert not ext.is_linear()
    for bad in (dict(intensities=np.ones((4, 4))), dict(total_intensity=np.ones(4)),
                dict(response=np.ones(3)), dict(photons_per_pixel=np.ones((4, 3)))):
        args = dict(mu_per_mm=mu, intensities=inten, total_intensity=inten.sum(0))
        args.update(bad)
        with pytest.raises(ValueError):
            ext.configure(P, 8, 6, **args)


def test_noisy_spectral_composition_tends_to_the_linear_case():
    """With very many photons the noisy loop approaches the linear formula, a bin
    without photons passes without noise, and the call count covers the live bins."""
    rng = np.random.default_rng(3)
    projs = rng.uniform(0.0, 40.0, (2, 2, 1, 6, 5)).astype(np.float32)
    mu = np.array([[0.0268, 0.0573], [0.0, 0.0], [0.0184, 0.0223]], np.float32)
    inten = np.array([[500.0, 600.0], [0.0, 0.0], [300.0, 200.0]])
    total = inten.sum(0)
    response = np.ones(3, np.float32)
    lin = np.zeros(projs.shape[1:])
    for b in (0, 2):
        lin += inten[b][:, None, None, None] * np.exp(-(projs[0] * mu[b, 0] + projs[1] * mu[b, 1]))
    lin = np.log(total[:, None, None, None] / lin)
    got, calls = _noisy_spectral_composition(projs, mu, inten, response, total, np.full((3, 1), 1e12, np.float32), 5)
    assert calls == 4
    assert rel_err(got, lin).max() < 1e-3
    quiet, _ = _noisy_spectral_composition(projs, mu, inten, response, total, np.zeros((3, 1), np.float32), 5)
    assert rel_err(quiet, lin).max() < 1e-5


@pytest.mark.gpu
def test_noisy_spectral_extension_matches_the_oracle_draw_for_draw(ctx):
    """SpectralEffectsExtension around projector | PoissonNoiseExtension: one batched
    projection of the material densities, then every (bin, material) noise draw and the
    combine in one kernel, against the reference loop composed from oracle pieces on the
    same material projections.  Bin 2 has no intensity (skipped, no nested call), bin 3
    no photons (passes without noise)."""
    import torch
    from ctl_b200 import geometry as G
    from ctl_b200 import phantom as Ph
    from ctl_b200.extensions import SpectralEffectsExtension
    from ctl_b200.projector import Settings, VoxelVolume
    vox = (2.0, 2.0, 2.0)
    water = Ph.ellipsoid_phantom((40, 40, 32), vox, 5, seed=41) * 40.0
    bone = Ph.ellipsoid_phantom((40, 40, 32), vox, 3, seed=42) * 20.0
    P = G.circular_flat(5, 750.0, 1000.0, G.FlatDetector(48, 40, 2.0, 2.0))
    mu = np.array([[0.0268, 0.0573], [0.0206, 0.0303], [0.0, 0.0], [0.0184, 0.0223]], np.float32)
    rng = np.random.default_rng(5)
    inten = rng.uniform(100.0, 1000.0, (4, 5))
    inten[2] = 0.0
    response = np.array([0.9, 0.95, 1.0, 0.8], np.float32)
    total = inten.sum(0)
    i0 = np.array([[2.0e4], [50.0], [1.0e3], [0.0]], np.float32)   # bin 1 low counts (inversion sampler)
    seed = 1234567
    ext = SpectralEffectsExtension(ctx)
    ext.configure(P, 48, 40, mu, inten, total, response, photons_per_pixel=i0, fixed_seed=seed)
    assert not ext.is_linear() and ext.nested_calls() == 6
    got = ext.project([VoxelVolume(water, vox), VoxelVolume(bone, vox)]).cpu().numpy()
    # the same material projections, through the single-call path (bitwise equal to the batch)
    projs = np.stack([ctx.project_volume(VoxelVolume(v, vox), P, 48, 40, Settings()) for v in (water, bone)])
    want, calls = _noisy_spectral_composition(projs, mu, inten, response, total, i0, seed)
    assert calls == 6
    finite = np.isfinite(want)
    assert (np.isfinite(got) == finite).all()
    close = np.isclose(got[finite], want[finite], rtol=1e-5, atol=1e-6)
    assert (~close).sum() <= 5, (~close).sum()   # a draw may flip on the last bit of an exp
    # the nested extension's next call draws anew; a fresh extension with the seed repeats
    again = ext.project([VoxelVolume(water, vox), VoxelVolume(bone, vox)]).cpu().numpy()
    assert ext.last_seed == seed + 6 and (again != got).mean() > 0.5
    ext2 = SpectralEffectsExtension(ctx)
    ext2.configure(P, 48, 40, mu, inten, total, response, photons_per_pixel=i0, fixed_seed=seed)
    np.testing.assert_array_equal(ext2.project([VoxelVolume(water, vox), VoxelVolume(bone, vox)]).cpu().numpy(),
                                  got)
    torch.cuda.synchronize()
    # the material volumes stayed resident across calls; release() frees them
    used = ctx.memory_used()
    ext.release()
    ext2.release()
    assert ctx.memory_used() < used


# ---- dynamic volumes ------------------------------------------------------------------------

def _dynamic_case():
    from ctl_b200 import geometry as G
    from ctl_b200 import phantom as Ph
    slope = Ph.ellipsoid_phantom((40, 40, 32), (2.0, 2.0, 2.0), 6, seed=31) * 0.5
    offset = Ph.ellipsoid_phantom((40, 40, 32), (2.0, 2.0, 2.0), 6, seed=32)
    P = G.circular_flat(6, 750.0, 1000.0, G.FlatDetector(48, 40, 2.0, 2.0))
    times = [0.0, 0.25, 0.5, 1.0, 1.7, 3.0]
    return slope, offset, P, times


def test_linear_dynamic_volume_matches_the_reference_update():
    """LinearDynamicVolume::updateVolume (img/lineardynamicvolume.cpp:194-198): slope * float(t) + offset."""
    from ctl_b200.extensions import LinearDynamicVolume
    slope, offset, _, _ = _dynamic_case()
    d = LinearDynamicVolume(slope, offset, (2.0, 2.0, 2.0))
    np.testing.assert_array_equal(d.at(1.7).data, slope * np.float32(1.7) + offset)


@pytest.mark.gpu
def test_dynamic_extension_matches_per_view_projection(ctx):
    """Every view equals the oracle's projection of the volume at that view's time
    (the reference's per-view loop), though it is computed by linearity from two
    batched projections."""
    from ctl_b200.extensions import DynamicProjectorExtension, LinearDynamicVolume
    from ctl_b200.projector import VoxelVolume
    slope, offset, P, times = _dynamic_case()
    ext = DynamicProjectorExtension(ctx)
    ext.configure(P, 48, 40, times)
    dyn = LinearDynamicVolume(slope, offset, (2.0, 2.0, 2.0))
    got = ext.project(dyn).cpu().numpy()
    for v, t in enumerate(times):
        want, _ = oracle.project_fp64(dyn.at(t).data, (2.0, 2.0, 2.0), P[v:v + 1], 48, 40)
        assert rel_err(got[v:v + 1], want).max() <= TOL, v
    # a volume that is not dynamic is projected as it is
    plain = ext.project(VoxelVolume(offset, (2.0, 2.0, 2.0))).cpu().numpy()
    want, _ = oracle.project_fp64(offset, (2.0, 2.0, 2.0), P, 48, 40)
    assert rel_err(plain, want).max() <= TOL
