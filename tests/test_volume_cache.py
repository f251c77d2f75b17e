"""The volume cache of ctlcu_project_volume (ctlcu_set_volume_cache).

The reference uploads the volume on every project() call
(raycasterprojector.cpp:239-269), and CTL's extensions call project() on one
volume many times (arealfocalspotextension.cpp:133-150,
spectraleffectsextension.cpp:385-391).  With the cache on, a volume seen
before -- the same description and the same voxels -- is projected from its
resident device copy; results must be bit-identical to uploading it again,
and any change to a voxel must be seen."""
import numpy as np
import pytest

from ctl_b200 import _lib as L
from ctl_b200 import geometry as G
from ctl_b200 import phantom as Ph
from ctl_b200.projector import (AcquisitionGeometry, Context, CudaRayCasterProjector, Settings, ViewDimensions,
                                VoxelVolume)


def test_cache_calls_need_a_context():
    lib = L.load()
    assert lib.ctlcu_set_volume_cache(None, 2) == L.ERR_INVALID_ARGUMENT
    assert lib.ctlcu_volume_cache_stats(None, None, None, None) == L.ERR_INVALID_ARGUMENT


def _case(seed=1):
    vol = Ph.ellipsoid_phantom((48, 40, 36), (2.0, 2.0, 2.0), 6, seed=seed)
    P = G.circular_flat(6, 750.0, 1000.0, G.FlatDetector(64, 48, 1.5, 1.5))
    return vol, P


@pytest.mark.gpu
def test_cached_projection_equals_upload_and_sees_changes():
    vol, P = _case()
    with Context(0) as plain, Context(0) as ctx:
        want = plain.project_volume(VoxelVolume(vol, (2.0, 2.0, 2.0)), P, 64, 48, Settings())
        ctx.set_volume_cache(2)
        first = ctx.project_volume(VoxelVolume(vol, (2.0, 2.0, 2.0)), P, 64, 48, Settings())
        again = ctx.project_volume(VoxelVolume(vol, (2.0, 2.0, 2.0)), P, 64, 48, Settings())
        st = ctx.volume_cache_stats()
        assert (st["hits"], st["misses"], st["resident"]) == (1, 1, 1)
        np.testing.assert_array_equal(first, want)
        np.testing.assert_array_equal(again, want)
        # one voxel changed in place: a miss, and the new content is projected
        vol2 = vol.copy()
        vol2[18, 20, 24] += 0.5
        got2 = ctx.project_volume(VoxelVolume(vol2, (2.0, 2.0, 2.0)), P, 64, 48, Settings())
        want2 = plain.project_volume(VoxelVolume(vol2, (2.0, 2.0, 2.0)), P, 64, 48, Settings())
        np.testing.assert_array_equal(got2, want2)
        assert not np.array_equal(got2, want)
        # the same voxels with another voxel size or offset are another volume
        got3 = ctx.project_volume(VoxelVolume(vol, (2.0, 2.0, 2.5)), P, 64, 48, Settings())
        want3 = plain.project_volume(VoxelVolume(vol, (2.0, 2.0, 2.5)), P, 64, 48, Settings())
        np.testing.assert_array_equal(got3, want3)
        st = ctx.volume_cache_stats()
        assert (st["hits"], st["misses"], st["resident"]) == (1, 3, 2)  # least recently used evicted
        # the first volume was the least recently used: projecting it again uploads it
        ctx.project_volume(VoxelVolume(vol, (2.0, 2.0, 2.0)), P, 64, 48, Settings())
        assert ctx.volume_cache_stats()["misses"] == 4
        # device-memory volumes bypass the cache
        import torch
        dvol = torch.from_numpy(vol).cuda()
        got_dev = ctx.project_volume(VoxelVolume(dvol, (2.0, 2.0, 2.0)), P, 64, 48, Settings())
        np.testing.assert_array_equal(got_dev, want)
        assert ctx.volume_cache_stats()["misses"] == 4
        # switching the cache off frees every resident copy
        ctx.set_volume_cache(0)
        assert ctx.volume_cache_stats()["resident"] == 0
        assert ctx.memory_used() == 0


@pytest.mark.gpu
def test_projector_reuses_the_volume_across_calls():
    """The CTL-facing projector keeps recent volumes resident by default, as an
    extension calling project() repeatedly on one volume would want."""
    vol, P = _case(3)
    p = CudaRayCasterProjector()
    p.configure(AcquisitionGeometry(P, ViewDimensions(64, 48, 1)))
    a = p.project(VoxelVolume(vol, (2.0, 2.0, 2.0))).numpy()
    b = p.project(VoxelVolume(vol, (2.0, 2.0, 2.0))).numpy()
    np.testing.assert_array_equal(a, b)
    st = p.context.volume_cache_stats()
    assert st["hits"] >= 1 and st["resident"] >= 1
    p.settings().volume_cache = 0
    c = p.project(VoxelVolume(vol, (2.0, 2.0, 2.0))).numpy()
    np.testing.assert_array_equal(a, c)
    assert p.context.volume_cache_stats()["resident"] == 0
