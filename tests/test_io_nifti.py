"""NIfTI-1 reader (io/nifti.rs read), host side: files written byte by byte here.

Each file is a 348-byte header plus voxels, written with struct.pack the way the
NIfTI-1 layout (nifti1.h) places every field; the reader's geometry is checked against
the LPS values the reference's reader forms (origin (−m03, −m13, m23), direction columns
(−m0d, −m1d, m2d) normalised, nifti.rs:1795-1876), its choice between the sform and the
quaternion form (the_mat, nifti.rs:1724-1768), its rescale (nifti.rs:2085-2099,
:2254-2300) and its refusals.
"""
import gzip
import os
import struct

import numpy as np
import pytest

from sitk_b200 import metric, _lib

DT = {np.uint8: 2, np.int16: 4, np.int32: 8, np.float32: 16, np.float64: 64, np.int8: 256, np.uint16: 512,
      np.uint32: 768, np.int64: 1024, np.uint64: 1280}


def header(shape_xyz, datatype, bitpix, *, pixdim=(1.0, 1.0, 1.0), qfac=1.0, dim0=3, extra_dims=(),
           vox_offset=352.0, scl=(0.0, 0.0), xyzt_units=2, qform=0, sform=0, quatern=(0.0, 0.0, 0.0),
           qoffset=(0.0, 0.0, 0.0), srow=None, intent=0, magic=b"n+1\0", big=False, sizeof_hdr=348):
    e = ">" if big else "<"
    dims = [dim0, *shape_xyz, *extra_dims]
    dims += [1] * (8 - len(dims))
    pd = [qfac, *pixdim] + [1.0] * 4
    b = bytearray(348)
    struct.pack_into(e + "i", b, 0, sizeof_hdr)
    struct.pack_into(e + "8h", b, 40, *dims)
    struct.pack_into(e + "h", b, 68, intent)
    struct.pack_into(e + "h", b, 70, datatype)
    struct.pack_into(e + "h", b, 72, bitpix)
    struct.pack_into(e + "8f", b, 76, *pd)
    struct.pack_into(e + "f", b, 108, vox_offset)
    struct.pack_into(e + "2f", b, 112, *scl)
    b[123] = xyzt_units
    struct.pack_into(e + "2h", b, 252, qform, sform)
    struct.pack_into(e + "6f", b, 256, *quatern, *qoffset)
    if srow is not None:
        struct.pack_into(e + "12f", b, 280, *np.asarray(srow, dtype=np.float64).ravel())
    b[344:348] = magic
    return bytes(b)


def nii_bytes(vol, **kw):
    """A single-file .nii of vol ([z, y, x]); header keywords as header()."""
    vol = np.ascontiguousarray(vol)
    big = kw.get("big", False)
    data = vol.astype(vol.dtype.newbyteorder(">" if big else "<")).tobytes()
    h = header((vol.shape[2], vol.shape[1], vol.shape[0]), DT[vol.dtype.type], vol.dtype.itemsize * 8, **kw)
    return h + b"\0" * 4 + data


def lps_geometry_of(m):
    """Origin and row-major direction the reference reader forms from a RAS matrix m."""
    m = np.asarray(m, dtype=np.float32).astype(np.float64)
    origin = np.array([-m[0, 3], -m[1, 3], m[2, 3]])
    d = np.zeros((3, 3))
    for c in range(3):
        ax = np.array([-m[0, c], -m[1, c], m[2, c]])
        d[:, c] = ax / np.linalg.norm(ax)
    return origin, d


def rotation(ax, ay, az):
    cx, sx, cy, sy, cz, sz = np.cos(ax), np.sin(ax), np.cos(ay), np.sin(ay), np.cos(az), np.sin(az)
    Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return Rz @ Rx @ Ry


def quatern_of(R):
    """(b, c, d) of a proper rotation R (a ≥ 0), from the unit-quaternion parametrisation
    R = [[a²+b²−c²−d², 2(bc−ad), 2(bd+ac)], [2(bc+ad), a²+c²−b²−d², 2(cd−ab)],
         [2(bd−ac), 2(cd+ab), a²+d²−b²−c²]]."""
    a = 0.5 * np.sqrt(max(1.0 + np.trace(R), 0.0))
    if a > 1e-3:
        return ((R[2, 1] - R[1, 2]) / (4 * a), (R[0, 2] - R[2, 0]) / (4 * a), (R[1, 0] - R[0, 1]) / (4 * a))
    b = 0.5 * np.sqrt(max(1.0 + R[0, 0] - R[1, 1] - R[2, 2], 0.0))
    return (b, (R[0, 1] + R[1, 0]) / (4 * b), (R[0, 2] + R[2, 0]) / (4 * b))


def write(tmp_path, name, blob, compress=False):
    p = tmp_path / name
    p.write_bytes(gzip.compress(blob) if compress else blob)
    return str(p)


def geo_arrays(g):
    return (np.array(g.size[:]), np.array(g.spacing[:]), np.array(g.origin[:]), np.array(g.direction[:]).reshape(3, 3))


def test_sform_scanner_anat_geometry_and_every_scalar_type(tmp_path):
    rng = np.random.default_rng(1)
    R = rotation(0.2, -0.1, 0.35)
    sp = np.array([0.8, 1.1, 2.5])
    o_ras = np.array([12.5, -30.25, 7.0])
    srow = np.zeros((3, 4))
    srow[:, :3] = R * sp
    srow[:, 3] = o_ras
    m = np.vstack([srow, [0, 0, 0, 1]])
    for dt in DT:
        info = np.iinfo(dt) if np.issubdtype(dt, np.integer) else None
        if info is not None:
            vol = rng.integers(max(info.min, -10 ** 6), min(info.max, 10 ** 6), size=(4, 5, 6)).astype(dt)
        else:
            vol = rng.normal(0, 100, size=(4, 5, 6)).astype(dt)
        p = write(tmp_path, f"v_{np.dtype(dt).name}.nii",
                  nii_bytes(vol, pixdim=tuple(sp), qform=1, sform=1, quatern=quatern_of(R), qoffset=tuple(o_ras),
                            srow=srow))
        out, g = metric.read_nifti_host(p)
        size, spacing, origin, direction = geo_arrays(g)
        np.testing.assert_array_equal(size, [6, 5, 4])
        np.testing.assert_allclose(spacing, sp.astype(np.float32), rtol=0, atol=0)
        eo, ed = lps_geometry_of(m)
        np.testing.assert_allclose(origin, eo, rtol=0, atol=1e-12)
        np.testing.assert_allclose(direction, ed, rtol=0, atol=1e-12)
        np.testing.assert_array_equal(out, vol.astype(np.float64).astype(np.float32))


def test_big_endian_and_gzip_and_upper_case_name(tmp_path):
    vol = np.arange(60, dtype=np.int16).reshape(3, 4, 5) - 20
    blob = nii_bytes(vol, big=True, pixdim=(1.5, 1.5, 3.0))
    for name, comp in (("be.nii", False), ("be.nii.gz", True), ("BE.NII.GZ", True)):
        out, g = metric.read_nifti_host(write(tmp_path, name, blob, compress=comp))
        np.testing.assert_array_equal(out, vol.astype(np.float32))
        assert list(g.spacing) == [1.5, 1.5, 3.0]
        # both codes unknown: origin 0 and the identity
        assert list(g.origin) == [0.0, 0.0, 0.0] and list(g.direction) == [1, 0, 0, 0, 1, 0, 0, 0, 1]


def test_scl_slope_and_inter_rescale_integers_through_f32(tmp_path):
    vol = np.array([[[-32768, -3, 0, 7, 32767]]], dtype=np.int16)
    out, _ = metric.read_nifti_host(write(tmp_path, "s.nii", nii_bytes(vol, scl=(0.25, -5.5))))
    expect = (vol.astype(np.float32).astype(np.float64) * 0.25 - 5.5).astype(np.float32)
    np.testing.assert_array_equal(out, expect)
    # a slope below DBL_EPSILON counts as 1: only the intercept applies
    out, _ = metric.read_nifti_host(write(tmp_path, "i.nii", nii_bytes(vol, scl=(0.0, 2.0))))
    np.testing.assert_array_equal(out, vol.astype(np.float32) + 2.0)
    # f64 data is rescaled in f64, then cast
    v64 = np.array([[[1.0 / 3.0, 2.5e10]]])
    out, _ = metric.read_nifti_host(write(tmp_path, "d.nii", nii_bytes(v64, scl=(3.0, 0.5))))
    np.testing.assert_array_equal(out, (v64 * 3.0 + 0.5).astype(np.float32))


def test_header_image_pair_and_analyze(tmp_path):
    vol = np.arange(24, dtype=np.uint8).reshape(2, 3, 4)
    h = header((4, 3, 2), 2, 8, vox_offset=0.0, magic=b"ni1\0", pixdim=(2.0, 2.0, 2.0))
    (tmp_path / "pair.hdr").write_bytes(h)
    (tmp_path / "pair.img").write_bytes(vol.tobytes())
    for name in ("pair.hdr", "pair.img"):
        out, g = metric.read_nifti_host(str(tmp_path / name))
        np.testing.assert_array_equal(out, vol.astype(np.float32))
        assert list(g.spacing) == [2.0, 2.0, 2.0]
    # the image file compressed beside a plain header
    (tmp_path / "gzpair.hdr").write_bytes(h)
    (tmp_path / "gzpair.img.gz").write_bytes(gzip.compress(vol.tobytes()))
    out, _ = metric.read_nifti_host(str(tmp_path / "gzpair.hdr"))
    np.testing.assert_array_equal(out, vol.astype(np.float32))
    # Analyze 7.5 (no magic): no rescale, no orientation, whatever the NIfTI fields hold
    ha = header((4, 3, 2), 2, 8, vox_offset=0.0, magic=b"\0\0\0\0", scl=(4.0, 1.0), qform=1, sform=1,
                srow=[[2, 0, 0, 9], [0, 2, 0, 9], [0, 0, 2, 9]])
    (tmp_path / "az.hdr").write_bytes(ha)
    (tmp_path / "az.img").write_bytes(vol.tobytes())
    out, g = metric.read_nifti_host(str(tmp_path / "az.img"))
    np.testing.assert_array_equal(out, vol.astype(np.float32))
    assert list(g.origin) == [0.0, 0.0, 0.0] and list(g.direction) == [1, 0, 0, 0, 1, 0, 0, 0, 1]


def test_quaternion_form_with_qfac_and_units(tmp_path):
    vol = np.zeros((2, 2, 2), dtype=np.float32)
    R = rotation(0.0, 0.0, np.pi / 2)
    q = quatern_of(R)
    for qfac in (1.0, -1.0):
        for units, scale in ((2, 1.0), (1, 1e3), (3, 1e-3)):
            blob = nii_bytes(vol, pixdim=(1.0, 2.0, 3.0), qfac=qfac, qform=2, quatern=q, qoffset=(4.0, 5.0, 6.0),
                             xyzt_units=units)
            _, g = metric.read_nifti_host(write(tmp_path, f"q{qfac}{units}.nii", blob))
            M = R.copy()
            if qfac < 0:
                M[:, 2] = -M[:, 2]
            m = np.eye(4)
            m[:3, :3] = M * np.array([1.0, 2.0, 3.0])
            m[:3, 3] = (4.0, 5.0, 6.0)
            eo, ed = lps_geometry_of(m)
            np.testing.assert_allclose(np.array(g.origin[:]), eo * scale, rtol=1e-12, atol=1e-12)
            np.testing.assert_allclose(np.array(g.direction[:]).reshape(3, 3), ed, rtol=0, atol=1e-6)
            np.testing.assert_allclose(np.array(g.spacing[:]), np.array([1.0, 2.0, 3.0]) * scale, rtol=1e-12)


def test_sform_or_quaternion_form_chosen_as_the_reference_chooses(tmp_path):
    vol = np.zeros((2, 2, 2), dtype=np.float32)
    Rq = rotation(0.0, 0.0, 0.3)
    q = quatern_of(Rq)
    qo = (1.0, 2.0, 3.0)
    Rs = rotation(0.4, 0.0, 0.0)
    srow = np.hstack([Rs, np.array([[7.0], [8.0], [9.0]])])
    m_s = np.vstack([srow, [0, 0, 0, 1]])
    m_q = np.eye(4)
    m_q[:3, :3] = Rq
    m_q[:3, 3] = qo
    cases = [
        # both aligned-anatomical and far apart: the quaternion form
        (2, 2, m_q),
        # the sform scanner-anatomical: the sform
        (2, 1, m_s),
        # no quaternion form: the sform
        (0, 2, m_s),
    ]
    for i, (qcode, scode, m) in enumerate(cases):
        blob = nii_bytes(vol, qform=qcode, sform=scode, quatern=q, qoffset=qo, srow=srow)
        _, g = metric.read_nifti_host(write(tmp_path, f"c{i}.nii", blob))
        eo, ed = lps_geometry_of(m)
        np.testing.assert_allclose(np.array(g.origin[:]), eo, rtol=0, atol=1e-6)
        np.testing.assert_allclose(np.array(g.direction[:]).reshape(3, 3), ed, rtol=0, atol=1e-6)
    # both aligned-anatomical and within the SVD comparison's 1e-4 of each other (distinct
    # spacings, so the singular bases are well defined): the sform
    sp = np.array([1.0, 2.0, 3.0])
    srow2 = np.hstack([Rq * sp, np.array(qo)[:, None]]) + 2e-6
    blob = nii_bytes(vol, pixdim=tuple(sp), qform=2, sform=2, quatern=q, qoffset=qo, srow=srow2)
    _, g = metric.read_nifti_host(write(tmp_path, "same.nii", blob))
    eo, _ = lps_geometry_of(np.vstack([srow2, [0, 0, 0, 1]]))
    np.testing.assert_allclose(np.array(g.origin[:]), eo, rtol=0, atol=1e-12)
    assert abs(g.origin[0] + 1.0) > 1e-6  # not the quaternion form's offset
    # a skewed sform with no quaternion form is refused (unless ITK_NIFTI_SFORM_PERMISSIVE)
    skew = np.array([[1.0, 0.5, 0.0, 0.0], [0.0, 1.0, 0.0, 0.0], [0.0, 0.0, 1.0, 0.0]])
    p = write(tmp_path, "skew.nii", nii_bytes(vol, sform=2, srow=skew))
    with pytest.raises(RuntimeError, match="MI_ERR_INVALID_ARGUMENT"):
        metric.read_nifti_host(p)


def test_trailing_unit_dimensions_and_refusals(tmp_path):
    vol = np.ones((2, 3, 4), dtype=np.float32)
    # a 4-D header whose fourth dimension is 1 is a 3-D volume
    blob = nii_bytes(vol, dim0=4, extra_dims=(1,))
    out, g = metric.read_nifti_host(write(tmp_path, "t1.nii", blob))
    assert list(g.size) == [4, 3, 2] and out.shape == (2, 3, 4)

    def refused(name, blob, status="MI_ERR_INVALID_ARGUMENT"):
        with pytest.raises(RuntimeError, match=status):
            metric.read_nifti_host(write(tmp_path, name, blob))

    refused("t2.nii", nii_bytes(np.ones((2, 3, 4), np.float32), dim0=4, extra_dims=(2,)))
    refused("two_d.nii", nii_bytes(np.ones((1, 3, 4), np.float32), dim0=2))
    refused("vec.nii", nii_bytes(vol, intent=1007))
    refused("trunc.nii", nii_bytes(vol)[:-8])
    refused("dt0.nii", header((4, 3, 2), 0, 32) + b"\0" * 100)
    refused("baddim.nii", header((4, 3, 2), 16, 32, dim0=9) + b"\0" * 200)
    c = header((4, 3, 2), 32, 64) + b"\0" * 4 + b"\0" * (24 * 8)
    refused("cplx.nii", c, "MI_ERR_UNSUPPORTED_PIXEL_TYPE")
    with pytest.raises(RuntimeError):
        metric.read_nifti_host(str(tmp_path / "missing.nii"))


def test_reader_exported():
    L = _lib.load()
    for name in ("mi_image_read_nifti", "mi_image_read_nifti_host"):
        assert hasattr(L, name)
