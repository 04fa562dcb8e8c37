"""The Mattes metric through a B-spline transform on the device vs the oracle's
sparse-support path (registration/mattes.rs:722-796), through the C ABI.

Contract: every sample's validity and both Parzen bins equal the oracle's exactly
(each sample takes the reference's exact FP64 chain); the value within 1e-5 relative;
each derivative component within 1e-4 of max|∂|; the derivative matches a central
finite difference of the device value.
"""
import ctypes

import numpy as np
import pytest

from conftest import small_pair

pytestmark = pytest.mark.gpu


def _setup(oracle, n, mesh, strategy=None, pct=1.0, seed=0, fmask=None, mmask=None, amp=0.8, spacing=(1.0, 1.0, 1.0),
           origin=(0.0, 0.0, 0.0), rseed=1):
    import sitk_b200 as sb
    from sitk_b200.transforms import BSplineTransform
    p = small_pair(n=n, seed=13, rot=6.0, trans=2.0)
    f = sb.DeviceImage.upload(p.fixed, spacing, origin)
    m = sb.DeviceImage.upload(p.moving, spacing, origin)
    metric = sb.DeviceMattesMetric.from_device_sampled(f, m, fixed_mask=fmask, moving_mask=mmask, bins=32,
                                                       strategy=strategy, percentage=pct, seed=seed)
    t = BSplineTransform.from_image_domain(f.geo, mesh)
    t.set_parameters(amp * np.random.default_rng(rseed).standard_normal(t.nparams))
    g = oracle.make_geometry((n, n, n), spacing, origin)
    draw = oracle.draw_samples(n ** 3, strategy, pct, seed) if strategy else None
    return p, metric, t, g, draw


def _records(metric, t):
    from sitk_b200 import _lib
    n = metric.sample_count()
    out = np.zeros(n, dtype=np.uint16)
    fp = np.ascontiguousarray(t.fixed_params)
    c = np.ascontiguousarray(t.params)
    dp = ctypes.POINTER(ctypes.c_double)
    _lib.check(_lib.load().mi_metric_bspline_records(metric.handle, fp.ctypes.data_as(dp), c.ctypes.data_as(dp),
                                                     c.size, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)), n),
               metric.ctx.handle)
    return out


def _compare(oracle, p, metric, t, g, draw, n, fmask=None, mmask=None):
    ref = oracle.bspline_mattes(p.fixed, g, p.moving, g, 32, t.fixed_params, t.params, fmask=fmask, mmask=mmask,
                                draw=draw, per_sample=True)
    # per-sample decisions, in the device's sample order: the same multiset of voxels,
    # matched voxel for voxel (repeated draws of one voxel have identical outcomes)
    oflat = np.arange(n ** 3) if draw is None else np.asarray(draw)
    if fmask is not None:
        oflat = oflat[np.asarray(fmask).ravel()[oflat] != 0]
    dev = metric.sample_order().astype(np.int64)
    o_ord = np.argsort(oflat, kind="stable")
    d_ord = np.argsort(dev, kind="stable")
    np.testing.assert_array_equal(oflat[o_ord], dev[d_ord])
    order = np.empty_like(o_ord)
    order[d_ord] = o_ord
    rec = _records(metric, t)
    st = ref["status"][order]
    np.testing.assert_array_equal(rec != 0, st == 2)
    ok = st == 2
    np.testing.assert_array_equal(rec[ok] & 0xff, ref["mi"][order][ok])
    np.testing.assert_array_equal(rec[ok] >> 8, ref["fi"][order][ok])
    mv = metric.evaluate(t)
    assert mv.valid_points == ref["valid"] > 0
    assert abs(mv.value - ref["value"]) <= 1e-5 * abs(ref["value"])
    scale = np.max(np.abs(ref["derivative"]))
    assert scale > 0
    assert np.max(np.abs(mv.derivative - ref["derivative"])) <= 1e-4 * scale
    assert metric.value(t) == mv.value
    return mv, ref


def test_bspline_full_grid(oracle_lib):
    p, metric, t, g, draw = _setup(oracle_lib, 36, (3, 3, 3))
    _compare(oracle_lib, p, metric, t, g, draw, 36)


def test_bspline_random_sampling_nonunit_geometry(oracle_lib):
    p, metric, t, g, draw = _setup(oracle_lib, 40, (4, 3, 5), strategy=2, pct=0.3, seed=77, spacing=(1.2, 0.9, 1.1),
                                   origin=(-4.0, 3.0, 2.0), rseed=4)
    _compare(oracle_lib, p, metric, t, g, draw, 40)


def test_bspline_with_masks(oracle_lib):
    rng = np.random.default_rng(6)
    fmask = (rng.random((32, 32, 32)) > 0.25).astype(np.uint8)
    mmask = (rng.random((32, 32, 32)) > 0.2).astype(np.uint8)
    p, metric, t, g, draw = _setup(oracle_lib, 32, (3, 3, 3), fmask=fmask, mmask=mmask, rseed=8)
    _compare(oracle_lib, p, metric, t, g, draw, 32, fmask=fmask, mmask=mmask)


def test_bspline_derivative_matches_central_difference(oracle_lib):
    p, metric, t, g, draw = _setup(oracle_lib, 32, (3, 3, 3), amp=0.5)
    an = metric.evaluate(t).derivative
    base = t.params.copy()
    h = 1e-3
    for k in np.argsort(-np.abs(an))[:8]:
        pp, pm = base.copy(), base.copy()
        pp[k] += h
        pm[k] -= h
        t.set_parameters(pp)
        vp = metric.value(t)
        t.set_parameters(pm)
        vm = metric.value(t)
        fd = (vp - vm) / (2 * h)
        assert abs(fd - an[k]) < 5e-3 * max(1.0, abs(an[k])), (k, fd, an[k])
    t.set_parameters(base)


def test_zero_field_equals_the_identity_affine():
    import sitk_b200 as sb
    from sitk_b200.transforms import BSplineTransform
    p = small_pair(n=30, seed=3)
    f = sb.DeviceImage.upload(p.fixed)
    m = sb.DeviceImage.upload(p.moving)
    metric = sb.DeviceMattesMetric.from_device(f, m, bins=32)
    t = BSplineTransform.from_image_domain(f.geo, (2, 2, 2))
    b = metric.evaluate(t)
    a = metric.evaluate(sb.TranslationTransform((0.0, 0.0, 0.0)))
    assert b.valid_points == a.valid_points
    assert abs(b.value - a.value) <= 1e-7 * abs(a.value)
