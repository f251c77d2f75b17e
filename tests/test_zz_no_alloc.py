"""ctlcu_project_noalloc, the projection entry point for callers that cannot
allocate device memory while they run, against ctlcu_project.

The no-allocation call keeps the per-(view, module) ray geometry in one
static device array instead of pool memory.  Its projections must equal those
of ctlcu_project on the same inputs, on two calls in a row that reuse that
array.  The file sorts last, so a run that stops at the first failure has run
every other test before it; it also passes alone in a fresh process, where its
first call looks up the array's device address.
"""
import ctypes

import numpy as np
import pytest

from ctl_b200 import _lib as L
from ctl_b200 import workloads as W
from ctl_b200.projector import Context, Settings, VoxelVolume
from tests._common import rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-4


@pytest.fixture(scope="module")
def job():
    import torch
    j = W.c1()  # 64^3 volume, 90 views of 128 x 128
    ctx = Context(0)
    vol = ctx.volume(VoxelVolume(j.volume, j.voxel))
    yield ctx, vol, j, torch
    ctx.close()


@pytest.mark.parametrize("kernel", [L.KERNEL_GATHER, L.KERNEL_CELLS, L.KERNEL_PAIRS],
                         ids=["gather", "cells", "pairs"])
def test_noalloc_matches_project_on_two_calls_in_a_row(job, kernel):
    ctx, vol, j, torch = job
    s = Settings(kernel=kernel)
    C_, R = j.channels, j.rows
    view_sets = [np.ascontiguousarray(j.pmats[0::2]), np.ascontiguousarray(j.pmats[1::2])]
    # ctlcu_project first: its result is the expectation, and it builds the
    # derived array (cells / pairs) that the no-allocation call reads
    want = [ctx.project(vol, P, C_, R, s) for P in view_sets]  # host pmats: synchronous
    keep = []
    for P in view_sets:  # back to back on one stream, sharing the scratch array
        dP = torch.from_numpy(P).cuda()
        out = torch.full((P.shape[0], P.shape[1], R, C_), -1.0, device="cuda")
        ctx.project_noalloc(vol, dP, out, s)
        keep.append((dP, out))
    torch.cuda.synchronize()
    ctx.sync()
    for (_, out), w in zip(keep, want):
        got = out.cpu().numpy()
        assert rel_err(got, w).max() <= TOL
        assert got.min() >= 0.0 and got.max() > 0.0


def test_noalloc_rejects_what_it_cannot_serve(job):
    ctx, vol, j, torch = job
    C_, R = j.channels, j.rows
    # more view-modules than the scratch array holds
    n = L.NOALLOC_MAX_VIEW_MODULES + 1
    dP = torch.from_numpy(np.repeat(j.pmats[:1], n, axis=0)).cuda()
    out = torch.empty((n, 1, 1, 1), device="cuda")
    with pytest.raises(L.CtlcuError) as e:
        ctx.project_noalloc(vol, dP, out, Settings(kernel=L.KERNEL_GATHER))
    assert e.value.status == L.ERR_INVALID_ARGUMENT and "scratch limit" in str(e.value)
    # host buffers would need staging memory: the binding refuses them before the
    # call, and the C ABI refuses them too
    P = np.ascontiguousarray(j.pmats[:2])
    host_out = np.zeros((2, 1, R, C_), np.float32)
    with pytest.raises(ValueError):
        ctx.project_noalloc(vol, P, host_out, Settings(kernel=L.KERNEL_GATHER))
    st = Settings(kernel=L.KERNEL_GATHER).to_c()
    rc = ctx.lib.ctlcu_project_noalloc(ctx.h, vol.handle, ctypes.byref(st), ctypes.c_void_p(P.ctypes.data), 2, 1,
                                       C_, R, ctypes.c_void_p(host_out.ctypes.data), None)
    assert rc == L.ERR_INVALID_ARGUMENT
    # buffers the kernel would index past: float32 matrices, an output of other views
    with pytest.raises(ValueError):
        ctx.project_noalloc(vol, torch.from_numpy(P).float().cuda(), torch.empty((2, 1, R, C_), device="cuda"))
    with pytest.raises(ValueError):
        ctx.project_noalloc(vol, torch.from_numpy(P).cuda(), torch.empty((3, 1, R, C_), device="cuda"))
    # a derived array that no earlier call built: the mean-voxel volume
    dP2 = torch.from_numpy(P).cuda()
    out2 = torch.empty((2, 1, R, C_), device="cuda")
    with pytest.raises(L.CtlcuError) as e:
        ctx.project_noalloc(vol, dP2, out2, Settings(volume_upsampling=0))
    assert e.value.status == L.ERR_INVALID_ARGUMENT and "not built" in str(e.value)
