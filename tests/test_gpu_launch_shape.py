"""Launch shapes (views per block, warp patch, rays per block, sample unroll):
every shape gives the same projection, the autotuner's choice serves later
calls, and bad shapes are refused.

A ray's samples and their order do not depend on which block or lane runs
it, so for one unroll every shape must give identical bits; the unroll only
regroups the FP32 partial sums, so the unrolls agree to rounding and each
stays within the 1e-4 bound of the FP64 oracle.
"""
import numpy as np
import pytest

import oracle
from ctl_b200 import _lib as L
from ctl_b200 import geometry as G
from ctl_b200 import phantom as Ph
from ctl_b200.projector import Context, Settings, VoxelVolume
from tests._common import rel_err

pytestmark = pytest.mark.gpu

SHAPES = [(b, v, lx) for b in (128, 256, 512) for v in (1, 2, 4) for lx in (4, 8) if (b, v, lx) != (128, 4, 4)]


def _job():
    # ragged on purpose: 7 views (a partial group for 2 and 4 views per block) and a
    # 37 x 29 detector (partial tiles of every width and height)
    vol = Ph.ellipsoid_phantom((36, 40, 32), (2.0, 2.0, 2.0), 6, seed=11)
    P = G.circular_flat(7, 700.0, 1100.0, G.FlatDetector(37, 29, 2.2, 2.2), angle_range=3.0,
                        rng=np.random.default_rng(4), jitter_mm=0.5, tilt_deg=0.3)
    return vol, P


def _multimodule():
    vol = Ph.ellipsoid_phantom((32, 32, 24), (3.0, 3.0, 3.0), 5, seed=12)
    P = G.helical_cylindrical(5, 1.0, 600.0, 1000.0, 3, 12, 10, 3.0, -20.0, 20.0)
    return vol, P


@pytest.mark.parametrize("kernel", [L.KERNEL_CELLS, L.KERNEL_PAIRS, L.KERNEL_GATHER])
def test_every_shape_gives_identical_bits(kernel):
    vol, P = _job()
    C, R = 37, 29
    want, _ = oracle.project_fp64(vol, (2.0, 2.0, 2.0), P, C, R)
    with Context(0) as ctx:
        h = ctx.volume(VoxelVolume(vol, (2.0, 2.0, 2.0)))
        base = ctx.project(h, P, C, R, Settings(kernel=kernel, block_rays=256, views_per_block=2, lanes_x=4,
                                                  unroll=4))
        assert rel_err(base, want).max() <= 1e-4
        for b, v, lx in SHAPES:
            got = ctx.project(h, P, C, R, Settings(kernel=kernel, block_rays=b, views_per_block=v, lanes_x=lx,
                                                     unroll=4))
            np.testing.assert_array_equal(got, base, err_msg=f"shape {b} rays / {v} views / lanes {lx}")
        h.release()


@pytest.mark.parametrize("kernel", [L.KERNEL_CELLS, L.KERNEL_PAIRS])
@pytest.mark.parametrize("unroll", [2, 8])
def test_unrolls_agree_and_stay_within_the_oracle_bound(kernel, unroll):
    vol, P = _job()
    C, R = 37, 29
    want, _ = oracle.project_fp64(vol, (2.0, 2.0, 2.0), P, C, R)
    with Context(0) as ctx:
        h = ctx.volume(VoxelVolume(vol, (2.0, 2.0, 2.0)))
        for accum in (L.ACCUM_FP64, L.ACCUM_KAHAN):
            base = ctx.project(h, P, C, R, Settings(kernel=kernel, accum=accum, unroll=4))
            got = ctx.project(h, P, C, R, Settings(kernel=kernel, accum=accum, unroll=unroll))
            assert rel_err(got, want).max() <= 1e-4
            np.testing.assert_allclose(got, base, rtol=2e-6, atol=1e-6 * np.abs(base).max())
            # and the shape still does not matter at this unroll
            other = ctx.project(h, P, C, R, Settings(kernel=kernel, accum=accum, unroll=unroll, block_rays=128,
                                                       views_per_block=4, lanes_x=8))
            np.testing.assert_array_equal(other, got)
        h.release()


@pytest.mark.parametrize("storage", [L.F32, L.BF16, L.F16])
def test_shapes_with_16bit_storage_nearest_upsampling_and_texture(storage):
    """Every sample loop shares the pixel mapping: non-default shapes give the default
    shape's bits for 16-bit storage, the nearest-voxel loop, up-sampled volumes and the
    texture filter too."""
    vol, P = _job()
    C, R = 37, 29
    forms = [Settings(), Settings(interpolate=False), Settings(volume_upsampling=2),
             Settings(interp_mode=L.INTERP_TEXTURE)]
    with Context(0) as ctx:
        h = ctx.volume(VoxelVolume(vol, (2.0, 2.0, 2.0)), storage)
        for s in forms:
            if storage == L.BF16 and s.interp_mode == L.INTERP_TEXTURE:
                continue   # texture filtering takes F32 and F16 storage only (no BF16 texture format)
            base = ctx.project(h, P, C, R, s)
            for b, v, lx in [(128, 4, 8), (512, 1, 4), (256, 4, 4)]:
                s2 = Settings(interpolate=s.interpolate, volume_upsampling=s.volume_upsampling,
                              interp_mode=s.interp_mode, block_rays=b, views_per_block=v, lanes_x=lx)
                np.testing.assert_array_equal(ctx.project(h, P, C, R, s2), base,
                                              err_msg=f"{s} with shape {b} rays / {v} views / lanes {lx}")
        h.release()


def test_multimodule_shapes_with_subrays():
    vol, P = _multimodule()
    C, R = 12, 10
    s0 = Settings(rays_per_pixel=[2, 1])
    want, _ = oracle.project_fp64(vol, (3.0, 3.0, 3.0), P, C, R, rays=(2, 1))
    with Context(0) as ctx:
        h = ctx.volume(VoxelVolume(vol, (3.0, 3.0, 3.0)))
        base = ctx.project(h, P, C, R, s0)
        assert rel_err(base, want).max() <= 1e-4
        for b, v, lx in [(128, 1, 4), (512, 4, 8), (256, 4, 4), (128, 2, 8)]:
            s = Settings(rays_per_pixel=[2, 1], block_rays=b, views_per_block=v, lanes_x=lx)
            np.testing.assert_array_equal(ctx.project(h, P, C, R, s), base)
        h.release()


def test_bad_shapes_are_refused():
    vol, P = _job()
    with Context(0) as ctx:
        h = ctx.volume(VoxelVolume(vol, (2.0, 2.0, 2.0)))
        for bad in (dict(block_rays=100), dict(block_rays=1024), dict(views_per_block=3), dict(lanes_x=16),
                    dict(unroll=3), dict(unroll=-1), dict(block_rays=128, views_per_block=4, lanes_x=4)):
            with pytest.raises(L.CtlcuError) as e:
                ctx.project(h, P, 37, 29, Settings(**bad))
            assert e.value.status == L.ERR_INVALID_ARGUMENT
        # a partly given shape is completed to a valid one (8x4 patches for an 8x4 tile)
        s = ctx.tuned_settings(h, 1, 37, 29, Settings(block_rays=128, views_per_block=4))
        assert (s.block_rays, s.views_per_block, s.lanes_x, s.unroll) == (128, 4, 8, 4)
        h.release()


def test_autotuned_shape_serves_later_calls():
    vol, P = _job()
    C, R = 37, 29
    with Context(0) as ctx:
        h = ctx.volume(VoxelVolume(vol, (2.0, 2.0, 2.0)))
        before = ctx.tuned_settings(h, 1, C, R)
        assert (before.kernel, before.block_rays, before.views_per_block, before.lanes_x, before.unroll) == \
            (L.KERNEL_CELLS, 256, 2, 4, 4)
        kernel, ms = ctx.autotune(h, P, C, R, max_views=4)
        assert all(t > 0 for t in ms.values())
        tuned = ctx.tuned_settings(h, 1, C, R)
        assert tuned.kernel == kernel
        assert tuned.block_rays in (128, 256, 512) and tuned.views_per_block in (1, 2, 4)
        assert tuned.lanes_x in (4, 8) and tuned.unroll in (2, 4, 8)
        # an automatic call runs exactly the tuned settings
        auto = ctx.project(h, P, C, R, Settings())
        explicit = ctx.project(h, P, C, R, tuned)
        np.testing.assert_array_equal(auto, explicit)
        want, _ = oracle.project_fp64(vol, (2.0, 2.0, 2.0), P, C, R)
        assert rel_err(auto, want).max() <= 1e-4
        # fields the caller sets stay as set
        pinned = ctx.tuned_settings(h, 1, C, R, Settings(unroll=8, block_rays=512))
        assert pinned.unroll == 8 and pinned.block_rays == 512
        # another detector size has no tuning: defaults
        other = ctx.tuned_settings(h, 1, C + 1, R)
        assert (other.block_rays, other.views_per_block, other.lanes_x, other.unroll) == (256, 2, 4, 4)
        h.release()


def test_plans_and_the_noalloc_call_run_the_given_shape():
    """A CUDA-graph plan (launched twice) and the no-allocation call, with a non-default
    shape, give the single call's bits with that shape."""
    import torch
    vol, P = _job()
    C, R = 37, 29
    with Context(0) as ctx:
        h = ctx.volume(VoxelVolume(vol, (2.0, 2.0, 2.0)))
        s = Settings(block_rays=128, views_per_block=4, lanes_x=8, unroll=8)
        alone = ctx.project(h, P, C, R, s)
        dP = torch.from_numpy(P).cuda()
        out = torch.zeros((P.shape[0], 1, R, C), device="cuda")
        torch.cuda.synchronize()
        plan = ctx.plan([(h, dP, out)], s)
        for _ in range(2):
            plan.launch()
            ctx.sync()
            np.testing.assert_array_equal(out.cpu().numpy(), alone)
            out.zero_()
            torch.cuda.synchronize()
        plan.close()
        out2 = torch.zeros_like(out)
        torch.cuda.synchronize()
        ctx.project_noalloc(h, dP, out2, s)
        ctx.sync()
        np.testing.assert_array_equal(out2.cpu().numpy(), alone)
        h.release()


def test_batch_runs_the_given_shape():
    import torch
    vol, P = _job()
    C, R = 37, 29
    with Context(0) as ctx:
        h = ctx.volume(VoxelVolume(vol, (2.0, 2.0, 2.0)))
        for shape in (dict(block_rays=128, views_per_block=4, lanes_x=8, unroll=8),
                      dict(block_rays=512, views_per_block=1, lanes_x=4, unroll=2)):
            s = Settings(**shape)
            alone = ctx.project(h, P, C, R, s)
            dP = torch.from_numpy(P).cuda()
            out = torch.zeros((P.shape[0], 1, R, C), device="cuda")
            ctx.project_batch([(h, dP, out)], s)
            ctx.sync()
            np.testing.assert_array_equal(out.cpu().numpy(), alone)
        h.release()
