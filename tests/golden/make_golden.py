"""Generate the golden fixtures in this directory from the reference itself.

    export CTL_REFERENCE_DIR=/root/reference   # the reference's source tree
    make -C oracle all ref          # builds oracle/_ref/libctlref.so from the reference sources
    python tests/golden/make_golden.py          # everything
    python tests/golden/make_golden.py den      # den_files.json only

Needs the reference sources, located by CTL_REFERENCE_DIR (only where this
script runs; the tests read the fixtures it writes, never the reference).

Writes
  geometry.npz     CTL's golden FullGeometry test data (testing/testData/tubeGeo.den,
                   cArmGeo.den: helical tube and C-arm wobble, 40 curved modules of
                   16 x 64 pixels, geometrytest.cpp:16-56) with, per view and module,
                   the packed QR and the source position computed by the reference's
                   own mat::QRdecomposition / ProjectionMatrix::sourcePosition and the
                   decomposeM sign rule (raycasterprojector.cpp:527-549)
  projections.npz  small seeded cases (volume, geometry, settings) with the output
                   of the reference's own ray_caster kernels
                   (raycasterprojector_interp.cl / _no_interp.cl run through
                   oracle/ref_harness.cpp)
  den_files.json   size, header and SHA-256 of testing/testData/tubeGeo.den and
                   cArmGeo.den (the DEN writer must reproduce them byte for byte)
  header.nrrd      testing/testData/header.nrrd, the reference's NRRD header test file
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from ctl_b200 import geometry as G  # noqa: E402
from ctl_b200 import phantom as Ph  # noqa: E402
from ctl_b200.den import read_full_geometry  # noqa: E402

REF = os.environ.get("CTL_REFERENCE_DIR")
if not REF:
    sys.exit("make_golden.py: set CTL_REFERENCE_DIR to the reference's source tree")
TESTDATA = os.path.join(REF, "testing", "testData")


def cases():
    """(name, volume args, geometry, settings) of the projection fixtures."""
    out = []
    det = G.FlatDetector(48, 40, 2.0, 2.0)
    P_circ = G.circular_flat(6, 750.0, 1000.0, det)
    vol32 = dict(shape=(32, 32, 32), voxel=(4.0, 4.0, 4.0), offset=(0.0, 0.0, 0.0), n_ell=6, seed=11)
    base = dict(rays=(1, 1), ray_sampling=0.3, upsampling=1, interpolate=True)
    out.append(("circ_interp", vol32, P_circ, 48, 40, base))
    out.append(("circ_nearest", vol32, P_circ, 48, 40, dict(base, interpolate=False)))
    out.append(("circ_rays2x3_up2", vol32, P_circ, 48, 40, dict(base, rays=(2, 3), upsampling=2)))
    out.append(("circ_up0", vol32, P_circ, 48, 40, dict(base, upsampling=0)))
    out.append(("circ_step1", vol32, P_circ, 48, 40, dict(base, ray_sampling=1.0)))
    # off-centre, anisotropic, non-cubic
    volaniso = dict(shape=(28, 20, 16), voxel=(3.0, 4.5, 6.0), offset=(12.0, -20.0, 7.5), n_ell=5, seed=5)
    jit = G.circular_flat(5, 750.0, 1200.0, G.FlatDetector(40, 36, 2.5, 2.5),
                          rng=np.random.default_rng(3), jitter_mm=0.5, tilt_deg=0.2)
    out.append(("aniso_offcentre", volaniso, jit, 40, 36, base))
    out.append(("aniso_nearest_rays3x2", volaniso, jit, 40, 36, dict(base, interpolate=False, rays=(3, 2))))
    # CTL's golden curved-detector geometries (first 2 views, 40 modules of 16 x 64)
    tube = read_full_geometry(os.path.join(TESTDATA, "tubeGeo.den"), 40)[:2]
    carm = read_full_geometry(os.path.join(TESTDATA, "cArmGeo.den"), 40)[:2]
    vol40 = dict(shape=(40, 40, 24), voxel=(2.0, 2.0, 2.0), offset=(0.0, 0.0, 0.0), n_ell=4, seed=7)
    out.append(("tube_modules", vol40, tube, 16, 64, base))
    out.append(("carm_modules", vol40, carm, 16, 64, base))
    return out


def main():
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref/libctlref.so is not built: make -C oracle ref")
    tube = read_full_geometry(os.path.join(TESTDATA, "tubeGeo.den"), 40)
    carm = read_full_geometry(os.path.join(TESTDATA, "cArmGeo.den"), 40)
    tq, ts = oracle.view_setup(tube, "ref")
    cq, cs = oracle.view_setup(carm, "ref")
    np.savez_compressed(os.path.join(HERE, "geometry.npz"), tube_pmats=tube, tube_qr=tq, tube_src=ts,
                        carm_pmats=carm, carm_qr=cq, carm_src=cs)

    arrays = {}
    meta = []
    for name, va, P, ch, rows, st in cases():
        vol = Ph.ellipsoid_phantom(va["shape"], va["voxel"], va["n_ell"], seed=va["seed"])
        ref = oracle.project_ref(vol, va["voxel"], P, ch, rows, offset_mm=va["offset"], rays=st["rays"],
                                 ray_sampling=st["ray_sampling"], upsampling=st["upsampling"],
                                 interpolate=st["interpolate"])
        arrays[f"{name}__volume"] = vol
        arrays[f"{name}__pmats"] = P
        arrays[f"{name}__ref"] = ref
        meta.append(dict(name=name, voxel=list(va["voxel"]), offset=list(va["offset"]), channels=ch,
                         rows=rows, rays=list(st["rays"]), ray_sampling=st["ray_sampling"],
                         upsampling=st["upsampling"], interpolate=st["interpolate"]))
        print(f"{name}: {ref.shape} max {ref.max():.4f}")
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "projections.npz"), **arrays)
    den_files()


def den_files():
    """den_files.json: size, header and SHA-256 of the reference's golden DEN files,
    so the DEN writer can be checked byte for byte without the files."""
    out = {}
    for name in ("tubeGeo.den", "cArmGeo.den"):
        raw = open(os.path.join(TESTDATA, name), "rb").read()
        out[name] = {"bytes": len(raw), "header": [int(v) for v in np.frombuffer(raw[:6], "<u2")],
                     "sha256": hashlib.sha256(raw).hexdigest()}
    with open(os.path.join(HERE, "den_files.json"), "w") as f:
        json.dump(out, f, indent=1)
    # the reference's NRRD reader test file (testing/src/nrrdfileiotest.cpp:6), copied as it is
    with open(os.path.join(TESTDATA, "header.nrrd"), "rb") as src, open(os.path.join(HERE, "header.nrrd"), "wb") as dst:
        dst.write(src.read())


if __name__ == "__main__":
    if sys.argv[1:] == ["den"]:
        den_files()
    else:
        main()
