"""The C++ CTL adapter (ctl_b200/adapter/, CTL::CUDA::CudaRayCasterProjector).

CTL and Qt are not available here, so the adapter is compiled against a
stand-in of the CTL/Qt headers it uses (tests/adapter/ctl_standin/, same class
and method names as CTL).  The CPU test checks that it compiles; the GPU test
links it with libctlcu.so and drives it through configure()/project() the way
CTL's extensions and pipelines do, against the oracle.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle
from tests._common import golden_cases, rel_err

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
STANDIN = os.path.join(HERE, "adapter", "ctl_standin")
ADAPTER = os.path.join(ROOT, "ctl_b200", "adapter")
FLAGS = ["-std=c++17", "-Wall", "-Werror", "-I", STANDIN, "-I", os.path.join(ROOT, "include"), "-I", ADAPTER]
SOURCES = [os.path.join(ADAPTER, "cudaraycasterprojector.cpp"), os.path.join(HERE, "adapter", "adapter_main.cpp")]

needs_gxx = pytest.mark.skipif(shutil.which("g++") is None, reason="g++ not available")


@needs_gxx
def test_adapter_compiles_against_the_ctl_interface(tmp_path):
    for src in SOURCES:
        obj = tmp_path / (os.path.basename(src) + ".o")
        r = subprocess.run(["g++", *FLAGS, "-c", src, "-o", str(obj)], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr


def _write_case(d, m, vol, P):
    nz, ny, nx = vol.shape
    V, M = P.shape[:2]
    with open(d / "meta.txt", "w") as f:
        f.write(" ".join(str(x) for x in (nx, ny, nz, *m["voxel"], *m["offset"], m["channels"], m["rows"], M, V,
                                          m["rays"][0], m["rays"][1], m["ray_sampling"], m["upsampling"],
                                          int(m["interpolate"]))))
    np.ascontiguousarray(vol, np.float32).tofile(d / "volume.bin")
    np.ascontiguousarray(P, np.float64).tofile(d / "pmats.bin")


@needs_gxx
@pytest.mark.gpu
def test_adapter_projects_through_ctl_interface_like_the_oracle(tmp_path):
    exe = tmp_path / "adapter_test"
    lib = os.path.join(ROOT, "ctl_b200")
    r = subprocess.run(["g++", *FLAGS, *SOURCES, "-L", lib, "-lctlcu", f"-Wl,-rpath,{lib}", "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    chosen = {"circ_interp", "circ_nearest", "circ_rays2x3_up2", "circ_up0", "aniso_offcentre", "tube_modules"}
    for m, vol, P, _ in (c for c in golden_cases() if c[0]["name"] in chosen):
        d = tmp_path / m["name"]
        d.mkdir()
        _write_case(d, m, vol, P)
        r = subprocess.run([str(exe), str(d)], capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, (m["name"], r.returncode, r.stderr)
        V, M = P.shape[:2]
        got = np.fromfile(d / "out.bin", np.float32).reshape(V, M, m["rows"], m["channels"])
        want, _ = oracle.project_fp64(vol, m["voxel"], P, m["channels"], m["rows"], offset_mm=m["offset"],
                                      rays=m["rays"], ray_sampling=m["ray_sampling"],
                                      upsampling=m["upsampling"], interpolate=m["interpolate"])
        tol = 3e-4 if (m["upsampling"] == 0 and m["interpolate"]) else 1e-4
        assert rel_err(got, want).max() <= tol, m["name"]
