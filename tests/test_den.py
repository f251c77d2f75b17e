"""DEN files through the C ABI (ctlcu_den_write / _header / _read).

Pinned to the reference's own golden DEN files: writing CTL's golden
geometries (tests/golden/geometry.npz) must reproduce testing/testData/tubeGeo.den
and cArmGeo.den byte for byte (their SHA-256, sizes and headers are in
tests/golden/den_files.json, recorded by tests/golden/make_golden.py).
"""
import hashlib
import json
import os

import numpy as np
import pytest

from ctl_b200 import _lib as L
from ctl_b200 import den as D
from tests._common import GOLDEN, golden_geometry


def _sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def test_writer_reproduces_the_reference_golden_files_byte_for_byte(tmp_path):
    ref = json.load(open(os.path.join(GOLDEN, "den_files.json")))
    g = golden_geometry()
    for key, name in (("tube", "tubeGeo.den"), ("carm", "cArmGeo.den")):
        p = tmp_path / name
        D.save_full_geometry(None, g[key + "_pmats"], p)
        assert os.path.getsize(p) == ref[name]["bytes"]
        assert list(D.header(p)[0]) == ref[name]["header"]
        assert _sha(p) == ref[name]["sha256"], name
        np.testing.assert_array_equal(D.load_full_geometry(None, p, 40), g[key + "_pmats"])


def test_numpy_and_c_writers_agree_for_every_element_type(tmp_path):
    rng = np.random.default_rng(0)
    for dt in (np.uint8, np.uint16, np.float32, np.float64):
        a = (rng.random((5, 7, 9)) * 200).astype(dt)
        D.write_den(tmp_path / "np.den", a)
        D.save(None, a, tmp_path / "c.den", 7, 9, 5)
        assert _sha(tmp_path / "np.den") == _sha(tmp_path / "c.den")
        assert D.header(tmp_path / "c.den") == ((7, 9, 5), np.dtype(dt).itemsize)
        np.testing.assert_array_equal(D.load(None, tmp_path / "c.den"), a)
        np.testing.assert_array_equal(D.load(None, tmp_path / "c.den", first=2, n=2), a[2:4])


def test_projections_round_trip_in_ctl_layout(tmp_path):
    p = np.random.default_rng(1).random((3, 2, 4, 6)).astype(np.float32)   # views, modules, rows, channels
    D.save_projections(None, p, tmp_path / "proj.den")
    assert D.header(tmp_path / "proj.den") == ((4, 6, 6), 4)   # rows, cols = channels, count = views x modules
    np.testing.assert_array_equal(D.load_projections(None, tmp_path / "proj.den", 2), p)


def test_reference_rules_are_enforced(tmp_path):
    lib = L.load()
    a = np.zeros(70000, np.float32)
    # a dimension above 65535 (gen_save: "exceeds 16 bit")
    assert lib.ctlcu_den_write(None, str(tmp_path / "x.den").encode(), a.ctypes.data, 4, 70000, 1, 1,
                               None) == L.ERR_INVALID_ARGUMENT
    assert lib.ctlcu_den_write(None, str(tmp_path / "x.den").encode(), a.ctypes.data, 3, 1, 1, 1,
                               None) == L.ERR_INVALID_ARGUMENT
    assert lib.ctlcu_den_write(None, str(tmp_path / "x.den").encode(), a.ctypes.data, 4, 0, 1, 1,
                               None) == L.ERR_INVALID_ARGUMENT
    # a header that does not match the data size
    with open(tmp_path / "bad.den", "wb") as f:
        f.write(np.array([2, 2, 2], "<u2").tobytes() + b"\0" * 7)
    with pytest.raises(L.CtlcuError):
        D.header(tmp_path / "bad.den")
    D.save(None, np.ones((2, 3, 4), np.float32), tmp_path / "ok.den", 3, 4, 2)
    with pytest.raises(L.CtlcuError):
        D.load(None, tmp_path / "ok.den", first=1, n=5)
    with pytest.raises(L.CtlcuError):
        D.load(None, tmp_path / "missing.den")


@pytest.mark.gpu
def test_device_data_streams_to_and_from_files(tmp_path):
    """Device tensors larger than the 32 MB staging buffers: the device path writes
    the same bytes as the host path and reads them back into device memory."""
    import torch
    from ctl_b200.projector import Context
    ctx = Context(0)
    try:
        V, M, R, Cn = 80, 1, 384, 512     # 63 MB: two staging buffers, several chunks each
        host = np.random.default_rng(2).random((V, M, R, Cn)).astype(np.float32)
        dev = torch.from_numpy(host).cuda()
        D.save_projections(ctx, dev, tmp_path / "dev.den")
        D.save_projections(None, host, tmp_path / "host.den")
        assert _sha(tmp_path / "dev.den") == _sha(tmp_path / "host.den")
        back = torch.empty_like(dev)
        D.load_projections(ctx, tmp_path / "dev.den", 1, out=back)
        assert torch.equal(back, dev)
        part = torch.empty((7, R, Cn), dtype=torch.float32, device="cuda")
        D.load(ctx, tmp_path / "dev.den", part, first=33, n=7)
        np.testing.assert_array_equal(part.cpu().numpy(), host[33:40, 0])
    finally:
        ctx.close()
