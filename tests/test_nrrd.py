"""NRRD files through the C ABI (ctlcu_nrrd_write_projections / _header / _read).

The reader is pinned to the reference's own NRRD test file (testing/testData/header.nrrd,
copied to tests/golden/ by make_golden.py) and the expectations of
testing/src/nrrdfileiotest.cpp:20-58.  The writer's header is the one that
NrrdFileIO::writeHeader produces for BaseTypeIO::write(ProjectionData)
(io/nrrd/nrrdfileio.tpp:252-337, io/basetypeio.tpp:342-362).
"""
import os

import numpy as np
import pytest

from ctl_b200 import _lib as L
from ctl_b200 import nrrd as N
from tests._common import GOLDEN


def test_reader_matches_the_reference_test_on_its_golden_header():
    h = N.header(os.path.join(GOLDEN, "header.nrrd"))
    assert h["version"] == 4
    assert h["sizes"] == [256, 256, 199]
    assert h["elem_bytes"] == 4
    assert h["offset"] == 118   # nrrdfileiotest.cpp:55-57: header offset 118


def test_writer_produces_ctls_projection_header_and_round_trips(tmp_path):
    p = np.random.default_rng(3).random((3, 2, 5, 7)).astype(np.float32)   # views, modules, rows, channels
    path = tmp_path / "proj.nrrd"
    N.save_projections(None, p, path)
    raw = open(path, "rb").read()
    expected = (b"NRRD0004\n"
                b"type: float\n"
                b"dimension: 4\n"
                b"sizes: 7 5 2 3\n"
                b'labels: "num channel" "num row" "num det module" "num proj"\n'
                b"encoding: raw\n"
                b"endian: little\n"
                b"type hint:=projection data\n"
                b"\n")
    assert raw[:len(expected)] == expected
    assert raw[len(expected):] == p.tobytes()
    h = N.header(path)
    assert h == {"version": 4, "sizes": [7, 5, 2, 3], "elem_bytes": 4, "offset": len(expected)}
    np.testing.assert_array_equal(N.load_projections(None, path), p)


@pytest.mark.parametrize("text,why", [
    (b"NRRX0004\ntype: float\n\n", "magic"),
    (b"NRRD0004\ntype: float\ndimension: 1\nsizes: 4\n", "no empty line"),
    (b"NRRD0004\ntype: float\ndimension: 5\nsizes: 1 1 1 1 1\n\n", "dimension"),
    (b"NRRD0004\ntype: float\ndimension: 2\nsizes: 4\n\n", "sizes count"),
    (b"NRRD0004\ntype: quaternion\ndimension: 1\nsizes: 4\n\n", "type"),
    (b"NRRD0004\ntype: float\ndimension: 1\nsizes: 4\nencoding: gzip\n\n", "encoding"),
    (b"NRRD0004\ntype: float\ndimension: 1\nsizes: 4\nthis is not a field\n\n", "entry"),
])
def test_invalid_headers_are_rejected(tmp_path, text, why):
    path = tmp_path / "bad.nrrd"
    path.write_bytes(text + b"\0" * 16)
    with pytest.raises(L.CtlcuError):
        N.header(path)


def test_comments_and_key_value_pairs_are_skipped(tmp_path):
    path = tmp_path / "c.nrrd"
    body = np.arange(6, dtype=np.float32)
    path.write_bytes(b"NRRD0004\n# a comment\ntype: float\n#another\nmy key:=x: y\ndimension: 2\n"
                     b"sizes: 3 2\nspacings: 1 1\nencoding: raw\nendian: little\n\n" + body.tobytes())
    h = N.header(path)
    assert h["sizes"] == [3, 2]
    out = np.empty(6, np.float32)
    L.check(L.load().ctlcu_nrrd_read(None, str(path).encode(), out.ctypes.data, out.nbytes, None))
    np.testing.assert_array_equal(out, body)


@pytest.mark.gpu
def test_device_projections_stream_to_and_from_nrrd(tmp_path):
    import torch
    from ctl_b200.projector import Context
    ctx = Context(0)
    try:
        host = np.random.default_rng(4).random((90, 1, 320, 384)).astype(np.float32)   # 44 MB
        dev = torch.from_numpy(host).cuda()
        N.save_projections(ctx, dev, tmp_path / "dev.nrrd")
        N.save_projections(None, host, tmp_path / "host.nrrd")
        assert open(tmp_path / "dev.nrrd", "rb").read() == open(tmp_path / "host.nrrd", "rb").read()
        back = torch.empty_like(dev)
        N.load_projections(ctx, tmp_path / "dev.nrrd", out=back)
        assert torch.equal(back, dev)
    finally:
        ctx.close()
