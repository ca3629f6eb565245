"""The .bgeo frame writer (replacement of OutputBego, FilesIO.cpp:6-24):
round trip through an independent reader of the Houdini classic layout."""
import struct

import numpy as np

from mpm_cuda_b200 import _lib as L


def read_bgeo(path: str) -> np.ndarray:
    """Reads the classic .bgeo layout: 'Bgeo' 'V' version, 8 counts, point
    attribute definitions, then each point as 4 big-endian floats plus its
    attributes.  Only files without extra attributes or primitives."""
    with open(path, "rb") as f:
        data = f.read()
    assert data[:4] == b"Bgeo" and data[4:5] == b"V"
    version, n_points, n_prims, n_pgroups, n_prgroups, n_pattr, n_vattr, n_prattr, n_dattr = \
        struct.unpack(">9i", data[5:41])
    assert version == 5 and n_prims == 0 and n_pattr == 0
    body = np.frombuffer(data[41:41 + 16 * n_points], dtype=">f4").reshape(n_points, 4)
    assert np.all(body[:, 3] == 1.0)
    assert data[41 + 16 * n_points:] == b"\x00\xff"
    return body[:, :3].astype(np.float32)


def test_bgeo_roundtrip(tmp_path):
    lib = L.load()
    rng = np.random.default_rng(0)
    x = rng.random((1000, 3)).astype(np.float32)
    p = str(tmp_path / "Frame000000.bgeo")
    assert lib.mpm_write_bgeo_positions(p.encode(), L.fptr(x), len(x)) == L.OK
    assert np.array_equal(read_bgeo(p), x)


def test_bgeo_empty_and_bad_path(tmp_path):
    lib = L.load()
    x = np.zeros((0, 3), np.float32)
    p = str(tmp_path / "empty.bgeo")
    assert lib.mpm_write_bgeo_positions(p.encode(), L.fptr(x), 0) == L.OK
    assert read_bgeo(p).shape == (0, 3)
    assert lib.mpm_write_bgeo_positions(b"/nonexistent-dir/x.bgeo", L.fptr(x), 0) == L.ERR_IO
    assert "cannot write" in L.last_error()
