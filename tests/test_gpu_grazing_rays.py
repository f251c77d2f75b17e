"""Rays that graze a face of the volume far from the origin of the index space.

A 520-voxel-tall volume has its top face 0.4 voxel below the plane of a circular scan,
so every ray runs through the outer half of the zero-padded layer above that face, at
z = 521.3 .. 521.5 in cell coordinates. There one FP32 rounding of an absolute sample
position is up to 3e-5 voxel. Carried into every sample of a ray, it moves these line
integrals by up to 5e-4 relative: emulating that form on the CPU gives 1459 of the
2048 pixels above 1e-4. So the sample loops must form positions relative to each
ray's integer origin to hold the 1e-4 bar against the FP64 oracle.
"""
import numpy as np
import pytest

import oracle
from ctl_b200 import _lib as L
from ctl_b200 import geometry as G
from ctl_b200.projector import Context, Settings, VoxelVolume
from tests._common import rel_err

pytestmark = pytest.mark.gpu

NZ = 520
OFFSET = (0.0, 0.0, -NZ / 2.0)  # top face at world z = 0
VOXEL = (1.0, 1.0, 1.0)
C, R = 32, 16


def _job():
    rng = np.random.default_rng(7)
    vol = rng.uniform(0.5, 1.5, (NZ, 24, 24)).astype(np.float32)
    # rows 0.02 mm apart at twice magnification: rays from 0.33 to 0.47 voxel above the face
    P = G.circular_flat(4, 300.0, 600.0, G.FlatDetector(C, R, 0.5, 0.02), z=0.4)
    return vol, P


@pytest.fixture(scope="module")
def oracle_result():
    vol, P = _job()
    want, _ = oracle.project_fp64(vol, VOXEL, P, C, R, offset_mm=OFFSET)
    assert (want > 0).all()  # every ray crosses the layer
    return vol, P, want


@pytest.mark.parametrize("accum", [L.ACCUM_KAHAN, L.ACCUM_FP64])
@pytest.mark.parametrize("kernel", [L.KERNEL_CELLS, L.KERNEL_PAIRS, L.KERNEL_GATHER])
def test_grazing_rays_far_from_the_origin(oracle_result, kernel, accum):
    vol, P, want = oracle_result
    with Context(0) as ctx:
        h = ctx.volume(VoxelVolume(vol, VOXEL, OFFSET))
        got = ctx.project(h, P, C, R, Settings(kernel=kernel, accum=accum))
        h.release()
    e = rel_err(got, want)
    assert e.max() <= 1e-4, f"max rel err {e.max():.2e}"
