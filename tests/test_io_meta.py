"""MetaImage reading (io/meta_image.rs read), host side (CPU) and through the device
upload (GPU).

The files are written here by hand, byte by byte, so the expected voxels and geometry
are known independently of the reader; the cases follow the reference's header rules:
a repeated key keeps its last value, origin and direction aliases resolve in MetaIO's
fixed order (and the legacy ones only at FileFormatVersion 0), booleans are true on a
leading T/t/1, big-endian data, a detached raw file, zlib and gzip payloads, and the
refusals (other dimensions, several channels, LIST, a LOCAL compressed header without
its size, truncated data).
"""
import gzip
import os
import zlib

import numpy as np
import pytest


def _write(path, header_lines, payload):
    with open(path, "wb") as f:
        f.write(("\n".join(header_lines) + "\n").encode())
        f.write(payload)


def _vol(dtype, shape=(5, 4, 3), seed=0):
    rng = np.random.default_rng(seed)
    if np.dtype(dtype).kind == "f":
        return (rng.standard_normal(shape) * 100).astype(dtype)
    info = np.iinfo(dtype)
    return rng.integers(max(info.min, -30000), min(info.max, 30000), size=shape, endpoint=True).astype(dtype)


def _read(path):
    from sitk_b200.metric import read_meta_host
    return read_meta_host(str(path))


def _geo_tuple(g):
    return ([int(g.size[i]) for i in range(3)], [g.spacing[i] for i in range(3)], [g.origin[i] for i in range(3)],
            [g.direction[i] for i in range(9)])


@pytest.mark.parametrize("etype,dtype", [("MET_UCHAR", np.uint8), ("MET_CHAR", np.int8), ("MET_USHORT", np.uint16),
                                         ("MET_SHORT", np.int16), ("MET_UINT", np.uint32), ("MET_INT", np.int32),
                                         ("MET_ULONG_LONG", np.uint64), ("MET_LONG", np.int64),
                                         ("MET_FLOAT", np.float32), ("MET_DOUBLE", np.float64)])
def test_every_scalar_type_local_little_endian(tmp_path, etype, dtype):
    v = _vol(dtype)
    p = tmp_path / "a.mha"
    _write(p, ["ObjectType = Image", "NDims = 3", "DimSize = 3 4 5", f"ElementType = {etype}",
               "ElementSpacing = 0.5 1.25 2", "Offset = -3 4.5 7", "ElementDataFile = LOCAL"], v.astype("<" + v.dtype.str[1:]).tobytes())
    vox, g = _read(p)
    np.testing.assert_array_equal(vox, v.astype(np.float64).astype(np.float32))
    assert _geo_tuple(g) == ([3, 4, 5], [0.5, 1.25, 2.0], [-3.0, 4.5, 7.0], [1, 0, 0, 0, 1, 0, 0, 0, 1])


def test_big_endian_detached_raw_and_direction(tmp_path):
    v = _vol(np.int16, (3, 6, 2), seed=3)
    (tmp_path / "pix.raw").write_bytes(v.astype(">i2").tobytes())
    p = tmp_path / "b.mhd"
    d = "0 -1 0 1 0 0 0 0 1"
    _write(p, ["NDims = 3", "DimSize = 2 6 3", "ElementType = MET_SHORT", "BinaryDataByteOrderMSB = True",
               f"TransformMatrix = {d}", "ElementDataFile = pix.raw"], b"")
    vox, g = _read(p)
    np.testing.assert_array_equal(vox, v.astype(np.float32))
    assert _geo_tuple(g)[3] == [0, -1, 0, 1, 0, 0, 0, 0, 1]


def test_alias_precedence_and_last_value_wins(tmp_path):
    v = _vol(np.float32, (2, 2, 2))
    p = tmp_path / "c.mha"
    # Origin beats Position beats Offset at version 0, whatever the line order; the
    # last TransformMatrix wins; ElementByteOrderMSB loses to BinaryDataByteOrderMSB
    _write(p, ["NDims = 3", "DimSize = 2 2 2", "Origin = 1 2 3", "Offset = 9 9 9", "Position = 5 5 5",
               "TransformMatrix = 1 0 0 0 0 1 0 1 0", "TransformMatrix = 1 0 0 0 1 0 0 0 1",
               "ElementByteOrderMSB = True", "BinaryDataByteOrderMSB = False", "ElementType = MET_FLOAT",
               "ElementDataFile = LOCAL"], v.astype("<f4").tobytes())
    vox, g = _read(p)
    np.testing.assert_array_equal(vox, v)
    assert _geo_tuple(g)[2] == [1.0, 2.0, 3.0]
    assert _geo_tuple(g)[3] == [1, 0, 0, 0, 1, 0, 0, 0, 1]
    # at FileFormatVersion 1 only Offset and TransformMatrix count
    q = tmp_path / "d.mha"
    _write(q, ["FileFormatVersion = 1", "NDims = 3", "DimSize = 2 2 2", "Origin = 1 2 3", "Offset = 9 8 7",
               "Orientation = 0 1 0 1 0 0 0 0 1", "ElementType = MET_FLOAT", "ElementDataFile = LOCAL"],
           v.astype("<f4").tobytes())
    _, g = _read(q)
    assert _geo_tuple(g)[2] == [9.0, 8.0, 7.0]
    assert _geo_tuple(g)[3] == [1, 0, 0, 0, 1, 0, 0, 0, 1]


def test_boolean_is_its_first_character(tmp_path):
    v = _vol(np.uint16, (2, 3, 2), seed=5)
    p = tmp_path / "e.mha"
    # "yes" is false (only T, t, 1 lead a true value), so little-endian
    _write(p, ["NDims = 3", "DimSize = 2 3 2", "ElementType = MET_USHORT", "BinaryDataByteOrderMSB = yes",
               "ElementDataFile = LOCAL"], v.astype("<u2").tobytes())
    vox, _ = _read(p)
    np.testing.assert_array_equal(vox, v.astype(np.float32))


@pytest.mark.parametrize("codec", ["zlib", "gzip"])
def test_compressed_local_and_detached(tmp_path, codec):
    v = _vol(np.float32, (4, 3, 5), seed=7)
    raw = v.astype("<f4").tobytes()
    z = zlib.compress(raw) if codec == "zlib" else gzip.compress(raw)
    p = tmp_path / "f.mha"
    _write(p, ["NDims = 3", "DimSize = 5 3 4", "ElementType = MET_FLOAT", "CompressedData = True",
               f"CompressedDataSize = {len(z)}", "ElementDataFile = LOCAL"], z)
    vox, _ = _read(p)
    np.testing.assert_array_equal(vox, v)
    (tmp_path / "g.zraw").write_bytes(z)
    q = tmp_path / "g.mhd"
    _write(q, ["NDims = 3", "DimSize = 5 3 4", "ElementType = MET_FLOAT", "CompressedData = 1",
               "ElementDataFile = g.zraw"], b"")
    vox, _ = _read(q)
    np.testing.assert_array_equal(vox, v)


@pytest.mark.parametrize("lines,payload", [
    (["NDims = 2", "DimSize = 2 2", "ElementType = MET_FLOAT", "ElementDataFile = LOCAL"], b"\0" * 16),
    (["NDims = 3", "DimSize = 2 2 2", "ElementType = MET_FLOAT", "ElementNumberOfChannels = 3",
      "ElementDataFile = LOCAL"], b"\0" * 96),
    (["NDims = 3", "DimSize = 2 2 2", "ElementType = MET_FLOAT", "ElementDataFile = LIST"], b"a.raw\n"),
    (["NDims = 3", "DimSize = 2 2 2", "ElementType = MET_FLOAT", "CompressedData = True",
      "ElementDataFile = LOCAL"], zlib.compress(b"\0" * 32)),
    (["NDims = 3", "DimSize = 2 2 2", "ElementType = MET_FLOAT", "ElementDataFile = LOCAL"], b"\0" * 31),
    (["NDims = 3", "DimSize = 2 2 2", "ElementType = MET_RGB", "ElementDataFile = LOCAL"], b"\0" * 32),
])
def test_refusals(tmp_path, lines, payload):
    from sitk_b200 import _lib
    p = tmp_path / "r.mha"
    _write(p, lines, payload)
    with pytest.raises(_lib.MiError):
        _read(p)


@pytest.mark.gpu
def test_device_read_matches_the_host_read(tmp_path):
    import sitk_b200 as sb
    v = _vol(np.int32, (6, 5, 4), seed=9)
    p = tmp_path / "h.mha"
    _write(p, ["NDims = 3", "DimSize = 4 5 6", "ElementType = MET_INT", "ElementSpacing = 1.5 1 0.75",
               "Offset = 1 2 3", "ElementDataFile = LOCAL"], v.astype("<i4").tobytes())
    img = sb.DeviceImage.read(str(p))
    host, g = _read(p)
    np.testing.assert_array_equal(img.to_host(), host)
    assert img.size == (4, 5, 6)
    assert [img.geo.spacing[i] for i in range(3)] == [1.5, 1.0, 0.75]
