"""The C ABI library: it loads, and exports exactly what include/ctlcu.h declares."""
import ctypes
import os
import re
import subprocess

import pytest

import ctl_b200
from ctl_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ctlcu.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"CTLCU_API\s+[\w\s\*]+?\b(ctlcu_\w+)\s*\(", text)))


def test_header_declares_the_boundary():
    syms = declared_symbols()
    for name in ("ctlcu_create", "ctlcu_destroy", "ctlcu_volume_create", "ctlcu_volume_release",
                 "ctlcu_project", "ctlcu_project_volume", "ctlcu_project_batch", "ctlcu_sync",
                 "ctlcu_last_error"):
        assert name in syms


def test_library_loads_and_exports_every_declared_symbol():
    lib = L.load()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert lib.ctlcu_abi_version() == L.ABI_VERSION == 2


def test_binding_covers_the_header():
    bound = {name for name, _, _ in L.SIGNATURES}
    assert bound == set(declared_symbols())


def test_only_the_c_abi_is_exported():
    out = subprocess.run(["nm", "-D", "--defined-only", L.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = sorted(line.split()[-1] for line in out.splitlines() if " T " in line)
    assert exported == declared_symbols()


def test_struct_layouts_match_the_header():
    assert ctypes.sizeof(L.VolumeDesc) == 3 * 4 + 3 * 4 + 3 * 4 + 4
    assert ctypes.sizeof(L.Settings) == 12 * 4
    assert ctypes.sizeof(L.Request) == 8 + 8 + 8 + 4 * 4


def test_struct_layouts_match_a_c_compiler(tmp_path):
    """sizeof and field offsets of every header struct, as gcc lays them out,
    against the ctypes binding."""
    structs = {"ctlcu_volume_desc": L.VolumeDesc, "ctlcu_settings": L.Settings, "ctlcu_request": L.Request,
               "ctlcu_detector_desc": L.DetectorDesc, "ctlcu_trajectory_desc": L.TrajectoryDesc}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "ctlcu.h"', "int main(void) {"]
    for cname, cls in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(line.rsplit(" ", 1) for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                               check=True).stdout.splitlines())
    for cname, cls in structs.items():
        assert int(got[cname]) == ctypes.sizeof(cls), cname
        for fname, _ in cls._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(cls, fname).offset, (cname, fname)


def test_default_settings_are_the_reference_defaults():
    s = L.load().ctlcu_settings_default()
    assert list(s.rays_per_pixel) == [1, 1]
    assert abs(s.ray_sampling - 0.3) < 1e-7
    assert s.volume_upsampling == 1 and s.interpolate == 1
    assert s.interp_mode == L.INTERP_SOFTWARE and s.accum == L.ACCUM_KAHAN
    # launch shape left to the autotuner / defaults
    assert (s.views_per_block, s.lanes_x, s.block_rays, s.unroll) == (0, 0, 0, 0)


def test_launch_shape_rules_mirror_the_kernel_tiling():
    """The tile of a shape is block/views pixels, 16 channels wide from 128 pixels
    up; a warp patch lanes_x x 32/lanes_x must tile it exactly (only 128 rays,
    4 views and 4x8 patches do not fit: an 8x4 tile)."""
    def tile(block, views):
        p = block // views
        tx = 16 if p >= 128 else 8
        return tx, p // tx
    bad = []
    for block in (128, 256, 512):
        for views in (1, 2, 4):
            tx, ty = tile(block, views)
            assert tx * ty == block // views
            for lanes in (4, 8):
                if ty % (32 // lanes) or tx % lanes:
                    bad.append((block, views, lanes))
                else:
                    warps = block // 32 // views
                    assert (tx // lanes) * (ty // (32 // lanes)) == warps
    assert bad == [(128, 4, 4)]


def test_bad_device_is_rejected_without_compute():
    lib = L.load()
    h = ctypes.c_void_p()
    assert lib.ctlcu_create(1 << 20, ctypes.byref(h)) == L.ERR_NO_DEVICE
    assert h.value is None


def test_null_arguments_are_rejected():
    lib = L.load()
    assert lib.ctlcu_create(0, None) == L.ERR_INVALID_ARGUMENT
    assert lib.ctlcu_destroy(None) == L.ERR_INVALID_ARGUMENT
    assert lib.ctlcu_sync(None) == L.ERR_INVALID_ARGUMENT


def test_package_exports():
    for name in ("CudaRayCasterProjector", "Context", "Settings", "VoxelVolume"):
        assert hasattr(ctl_b200, name)
