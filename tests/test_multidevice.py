"""Several devices behind one projection: RayCasterProjector::Settings::deviceIDs
(raycasterprojector.h:30) through ctlcu_group_* and the adapters.

The reference deals views out round-robin over min(#deviceIDs, #views)
devices with the volume replicated on each (raycasterprojector.cpp:188,
:239-251, :321-357); here each device takes a contiguous block of views
(ctlcu_split_views).  The CPU tests pin the split; the GPU tests list one GPU
several times ({0, 0}, {0, 0, 0}: several contexts, streams and host threads on
one device), which must give the same bits as a one-device call.
"""
import numpy as np
import pytest

from ctl_b200 import _lib as L


@pytest.mark.parametrize("n_views,n_parts", [(360, 1), (360, 8), (361, 8), (90, 7), (5, 3), (3, 8), (0, 4),
                                             (1440, 3)])
def test_view_split_is_contiguous_balanced_and_complete(n_views, n_parts):
    first = L.split_views(n_views, n_parts)
    assert len(first) == n_parts + 1 and first[0] == 0 and first[-1] == n_views
    sizes = np.diff(first)
    assert (sizes >= 0).all() and sizes.max() - sizes.min() <= 1
    # the larger blocks come first
    assert list(sizes) == sorted(sizes, reverse=True)


def test_rank_shards_follow_the_library_split():
    """bench.py's ranks and ctl_b200.sharding take the blocks ctlcu_split_views gives."""
    from ctl_b200.sharding import shard_views
    for n_views, world in [(360, 8), (361, 3), (90, 7), (5, 8), (1440, 6)]:
        first = L.split_views(n_views, world)
        assert [shard_views(n_views, world, r) for r in range(world)] == \
            [(first[r], first[r + 1]) for r in range(world)]


def test_view_split_refuses_no_parts():
    lib = L.load()
    import ctypes as C
    first = (C.c_uint32 * 2)()
    assert lib.ctlcu_split_views(10, 0, first) == L.ERR_INVALID_ARGUMENT
    assert lib.ctlcu_split_views(10, 1, None) == L.ERR_INVALID_ARGUMENT


def test_group_without_a_device_fails_cleanly():
    """A device ordinal that does not exist is an error (raycasterprojector.cpp:442-447),
    reported as a status, not a crash; without any GPU every group creation fails so."""
    import ctypes as C
    lib = L.load()
    h = C.c_void_p()
    bad = (C.c_int * 1)(4096)
    assert lib.ctlcu_group_create(bad, 1, C.byref(h)) == L.ERR_NO_DEVICE
    assert not h.value
    if L.device_count() == 0:
        assert lib.ctlcu_group_create(None, 0, C.byref(h)) == L.ERR_NO_DEVICE


def _c1_case(n_views=90):
    from ctl_b200 import workloads as W
    job = W.c1()
    return job.volume, job.voxel, job.pmats[:n_views], job.channels, job.rows


@pytest.mark.gpu
@pytest.mark.parametrize("devices", [[0], [0, 0], [0, 0, 0]])
def test_group_equals_one_device_bit_for_bit(devices):
    from ctl_b200.projector import Context, Group, Settings, VoxelVolume
    vol, voxel, P, C, R = _c1_case()
    with Context(0) as ctx:
        want = ctx.project_volume(VoxelVolume(vol, voxel), P, C, R, Settings())
    with Group(devices) as g:
        assert g.size() == len(devices)
        got = g.project_volume(VoxelVolume(vol, voxel), P, C, R, Settings())
    np.testing.assert_array_equal(got, want)


@pytest.mark.gpu
def test_group_with_more_devices_than_views():
    """min(#devices, #views) devices take part (raycasterprojector.cpp:188)."""
    from ctl_b200.projector import Context, Group, Settings, VoxelVolume
    vol, voxel, P, C, R = _c1_case(2)
    with Context(0) as ctx:
        want = ctx.project_volume(VoxelVolume(vol, voxel), P, C, R, Settings())
    with Group([0, 0, 0, 0]) as g:
        got = g.project_volume(VoxelVolume(vol, voxel), P, C, R, Settings())
    np.testing.assert_array_equal(got, want)


@pytest.mark.gpu
def test_group_reports_the_failing_device():
    from ctl_b200.projector import Group, Settings, VoxelVolume
    vol, voxel, P, C, R = _c1_case(4)
    with Group([0, 0]) as g:
        with pytest.raises(L.CtlcuError) as e:
            g.project_volume(VoxelVolume(vol, voxel), P, C, R, Settings(ray_sampling=0.0))
        assert e.value.status == L.ERR_INVALID_ARGUMENT
        assert "device 0 of the group (cuda:0)" in str(e.value)
        # the group stays usable
        assert np.isfinite(g.project_volume(VoxelVolume(vol, voxel), P, C, R, Settings())).all()


@pytest.mark.gpu
def test_projector_device_ids():
    """The Python mirror of the adapter: settings().device_ids = [0, 0] through a group."""
    from ctl_b200.projector import (AcquisitionGeometry, CudaRayCasterProjector, ViewDimensions, VoxelVolume)
    vol, voxel, P, C, R = _c1_case(30)
    p = CudaRayCasterProjector()
    p.configure(AcquisitionGeometry(P, ViewDimensions(C, R, 1)))
    one = p.project(VoxelVolume(vol, voxel)).numpy()
    seen = []
    p.notifier.append(seen.append)
    p.settings().device_ids = [0, 0]
    two = p.project(VoxelVolume(vol, voxel)).numpy()
    np.testing.assert_array_equal(two, one)
    assert seen == list(range(30))
    p.settings().device_ids = [4096]
    with pytest.raises(L.CtlcuError):
        p.project(VoxelVolume(vol, voxel))
