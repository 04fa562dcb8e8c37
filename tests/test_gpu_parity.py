"""Device metric vs the CPU oracle, through the C ABI (needs a B200).

Contract (the reference's own device pins, tests/mattes_device.rs:189-350): every
sample's validity and both Parzen bins equal the oracle's exactly; the value is
within 1e-5 relative; each derivative component is within 1e-4 of max|∂| (the
reference scales its derivative band by max|∂|, tests/mattes_device.rs:337-350).
"""
import numpy as np
import pytest

from conftest import small_pair

pytestmark = pytest.mark.gpu

VALUE_RTOL = 1e-5
DERIV_RTOL = 1e-4


def _sb():
    import sitk_b200
    return sitk_b200


def _upload_pair(p, spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0)):
    sb = _sb()
    f = sb.DeviceImage.upload(p.fixed, spacing, origin)
    m = sb.DeviceImage.upload(p.moving, spacing, origin)
    return f, m


def _oracle_geo(oracle, n, spacing, origin):
    return oracle.make_geometry((n, n, n), spacing=spacing, origin=origin)


def bf16_round(v):
    """f32 → nearest BF16 (ties to even), widened back to f32 (finite inputs)."""
    b = np.ascontiguousarray(v, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(np.shape(v))


def _compare(oracle, p, n, transform, bins, spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0),
             strategy=None, pct=1.0, seed=0, mmask=None, fmask=None, explicit=None, moving_storage="f32",
             nthreads=1, other_form=True):
    """With moving_storage "bf16" the oracle runs on the moving volume rounded to BF16
    (the values the device metric samples), so the same exact contract applies.
    other_form=False skips the comparison with the other launch form."""
    sb = _sb()
    f, m = _upload_pair(p, spacing, origin)
    if moving_storage == "bf16":
        import dataclasses
        p = dataclasses.replace(p, moving=bf16_round(p.moving))
    kw = {}
    draw = None
    if explicit is not None:
        draw = np.asarray(explicit, dtype=np.int64)
    elif strategy is not None:
        draw = oracle.draw_samples(n ** 3, strategy, pct, seed)
    metric = sb.DeviceMattesMetric.from_device_sampled(
        f, m, fixed_mask=fmask, moving_mask=mmask, samples=explicit, bins=bins,
        strategy=strategy, percentage=pct, seed=seed, moving_storage=moving_storage)
    g = _oracle_geo(oracle, n, spacing, origin)
    ref = oracle.evaluate(p.fixed, g, p.moving, g, bins, transform.kind, transform.params,
                          transform.fixed_params, fmask=fmask, mmask=mmask, draw=draw,
                          per_sample=True, nthreads=nthreads)
    info = metric.info()
    ginfo = oracle.geometry_info(p.fixed, g, p.moving, g, bins, fmask=fmask, mmask=mmask, draw=draw)
    for k in ("fixed_min", "fixed_max", "moving_min", "moving_max", "fixed_bin_size", "moving_bin_size",
              "fixed_normalized_min", "moving_normalized_min"):
        assert info[k] == ginfo[k], k
    assert info["n_samples"] == ginfo["nsamples"]

    # exact per-sample decisions, in the device's sample order (the same multiset of
    # voxels; matched voxel for voxel, since equal voxels give equal decisions)
    st = sb.transform_stage(transform)
    dec = metric.sample_decisions(st)
    if draw is None and fmask is None:
        oflat = np.arange(n ** 3)
    else:
        oflat = np.arange(n ** 3) if draw is None else draw
        if fmask is not None:
            oflat = oflat[np.asarray(fmask).ravel()[oflat] != 0]
    dev = np.asarray(dec["flat"], dtype=np.int64)
    np.testing.assert_array_equal(dev, metric.sample_order())
    o_ord = np.argsort(oflat, kind="stable")
    d_ord = np.argsort(dev, kind="stable")
    np.testing.assert_array_equal(dev[d_ord], oflat[o_ord])
    order = np.empty_like(o_ord)
    order[d_ord] = o_ord
    o_status = ref["status"][order]
    np.testing.assert_array_equal(dec["status"], o_status)
    np.testing.assert_array_equal(dec["fi"], np.where(o_status == 2, ref["fi"][order], -1))
    np.testing.assert_array_equal(dec["mi"], np.where(o_status == 2, ref["mi"][order], -1))

    mv = metric.evaluate(transform)
    assert mv.valid_points == ref["valid"]
    assert abs(mv.value - ref["value"]) <= VALUE_RTOL * abs(ref["value"])
    scale = np.max(np.abs(ref["derivative"]))
    assert np.max(np.abs(mv.derivative - ref["derivative"])) <= DERIV_RTOL * scale, (mv.derivative, ref["derivative"])
    # value-only path agrees with evaluate
    v = metric.value(transform)
    assert v == mv.value
    if not other_form:
        return metric, mv, ref, dec
    # the split launch form (two kernels) computes the same histogram and tail, so
    # the same value bits; its derivative sums the moments over another partition of
    # the samples (FP32 within a thread, FP64 from the warp on), so the two forms agree
    # to FP32 accumulation error
    from sitk_b200.metric import get_fused, set_fused
    fused = get_fused(metric)
    set_fused(metric, not fused)
    other = metric.evaluate(transform)
    assert metric.value(transform) == mv.value
    set_fused(metric, fused)
    assert other.value == mv.value and other.valid_points == mv.valid_points
    np.testing.assert_allclose(other.derivative, mv.derivative, rtol=0, atol=1e-6 * max(scale, 1e-300))
    return metric, mv, ref, dec


def test_affine_full_grid_config0_shape(oracle_lib):
    sb = _sb()
    from sitk_b200 import synth
    p = synth.config0_pair()
    c = [31.5] * 3
    t = sb.AffineTransform(np.eye(3) + 0.01 * np.array([[1, 2, 0], [0, -1, 1], [1, 0, 2]]), (0.5, -0.3, 0.2), c)
    _compare(oracle_lib, p, 64, t, 50)


def test_versor_random_sampling(oracle_lib):
    sb = _sb()
    p = small_pair(n=48, seed=21, rot=12.0, trans=6.0, scale=None)
    t = sb.VersorRigid3DTransform((0.02, -0.03, 0.01), (0.7, -0.4, 0.9), [23.5] * 3)
    _, _, _, dec = _compare(oracle_lib, p, 48, t, 32, strategy=2, pct=0.1, seed=20261203)
    # the fast path decides almost every sample; the exact chain takes the rest
    assert dec["exact"].mean() < 0.02


def test_euler_regular_sampling_nonunit_geometry(oracle_lib):
    sb = _sb()
    p = small_pair(n=40, seed=4)
    sp, org = (1.2, 0.9, 1.1), (-10.0, 4.0, 2.5)
    c = [org[d] + sp[d] * 19.5 for d in range(3)]
    t = sb.Euler3DTransform((0.03, -0.02, 0.05), (0.4, 0.2, -0.6), c)
    _compare(oracle_lib, p, 40, t, 64, spacing=sp, origin=org, strategy=1, pct=0.25)


def test_masks_and_explicit_samples(oracle_lib):
    sb = _sb()
    p = small_pair(n=32, seed=8)
    rng = np.random.default_rng(5)
    mmask = (rng.random(p.moving.shape) > 0.1).astype(np.uint8)
    fmask = (rng.random(p.fixed.shape) > 0.3).astype(np.float32)
    explicit = rng.integers(0, 32 ** 3, size=9000)
    t = sb.AffineTransform(np.eye(3), (0.3, 0.1, -0.2), [15.5] * 3)
    _compare(oracle_lib, p, 32, t, 50, mmask=mmask, fmask=fmask, explicit=explicit)


def test_commensurate_identity_puts_samples_on_bin_edges(oracle_lib):
    # tests/mattes_device.rs:88-101: integer-valued volumes at the identity pose put
    # many Parzen terms exactly on integers — the exactness contract's hardest case.
    sb = _sb()
    rng = np.random.default_rng(2)
    n = 24
    vol = rng.integers(0, 47, size=(n, n, n)).astype(np.float32)
    vol[0, 0, 0] = 0.0
    vol[-1, -1, -1] = 46.0

    class P:
        fixed = vol
        moving = vol

    t = sb.TranslationTransform((0.0, 0.0, 0.0))
    metric, mv, ref, dec = _compare(oracle_lib, P, n, t, 50)
    assert ref["valid"] == n ** 3
    assert dec["exact"].mean() > 0.5  # bin edges everywhere: the exact chain decides


def test_boundary_straddle_translation(oracle_lib):
    # half-voxel shifts put continuous indices exactly on −0.5 / size−0.5
    sb = _sb()
    p = small_pair(n=20, seed=3)
    for tx in (0.5, -0.5, 0.25):
        t = sb.TranslationTransform((tx, -tx, 0.5))
        _compare(oracle_lib, p, 20, t, 40)


def test_degenerate_when_nothing_overlaps(oracle_lib):
    sb = _sb()
    p = small_pair(n=16, seed=1)
    f, m = _upload_pair(p)
    metric = sb.DeviceMattesMetric.from_device(f, m, 32)
    mv = metric.evaluate(sb.TranslationTransform((1000.0, 0.0, 0.0)))
    assert mv.valid_points == 0
    assert mv.value == np.finfo(np.float64).max
    assert np.all(mv.derivative == 0.0)


def test_repeated_evaluations_are_bit_identical():
    sb = _sb()
    p = small_pair(n=40, seed=12)
    f, m = _upload_pair(p)
    metric = sb.DeviceMattesMetric.from_device_sampled(f, m, bins=50, strategy=2, percentage=0.5, seed=9)
    t = sb.AffineTransform(np.eye(3) * 1.01, (0.2, 0.3, 0.1), [19.5] * 3)
    a = metric.evaluate(t)
    for _ in range(3):
        b = metric.evaluate(t)
        assert a.value == b.value and a.valid_points == b.valid_points
        np.testing.assert_array_equal(a.derivative, b.derivative)


def test_refusals_are_named():
    sb = _sb()
    p = small_pair(n=16, seed=1)
    f, m = _upload_pair(p)
    with pytest.raises(sb.MiError) as e:
        sb.DeviceMattesMetric.from_device(f, m, 4)
    assert e.value.name == "MI_ERR_TOO_FEW_HISTOGRAM_BINS"
    with pytest.raises(sb.MiError) as e:
        sb.DeviceMattesMetric.from_device(f, m, 1000)
    assert e.value.name == "MI_ERR_TOO_MANY_HISTOGRAM_BINS"
    c = sb.DeviceImage.upload(np.full((16, 16, 16), 5.0, dtype=np.float32))
    with pytest.raises(sb.MiError) as e:
        sb.DeviceMattesMetric.from_device(c, m, 32)
    assert e.value.name == "MI_ERR_CONSTANT_FIXED"
    with pytest.raises(sb.MiError) as e:
        sb.DeviceMattesMetric.from_device(f, c, 32)
    assert e.value.name == "MI_ERR_CONSTANT_MOVING"
    with pytest.raises(sb.MiError) as e:
        sb.DeviceMattesMetric.from_device_sampled(f, m, samples=[0, 5, 16 ** 3], bins=32)
    assert e.value.name == "MI_ERR_SAMPLE_INDEX_OUT_OF_GRID"
    with pytest.raises(sb.MiError) as e:
        sb.DeviceMattesMetric.from_device_sampled(f, m, fixed_mask=np.ones((8, 8, 8), np.float32), bins=32)
    assert e.value.name == "MI_ERR_MASK_SIZE_MISMATCH"
    sing = sb.DeviceImage.upload(p.moving, direction=(1, 0, 0, 1, 0, 0, 0, 0, 1))
    with pytest.raises(sb.MiError) as e:
        sb.DeviceMattesMetric.from_device(f, sing, 32)
    assert e.value.name == "MI_ERR_SINGULAR_DIRECTION"
    metric = sb.DeviceMattesMetric.from_device(f, m, 32)
    for bad in (np.zeros(0), np.zeros(12 * 9)):
        with pytest.raises(sb.MiError) as e:
            metric.value_stages(bad)
        assert e.value.name == "MI_ERR_POINT_MAP_STAGE_COUNT"
    with pytest.raises(sb.MiError) as e:
        sb.DeviceImage.upload(np.zeros((4, 4, 4), dtype=np.complex64))
    assert e.value.name == "MI_ERR_UNSUPPORTED_PIXEL_TYPE"
    # an unknown texture layout is refused through the C ABI options
    import ctypes
    from sitk_b200 import _lib
    opts = _lib.MiMetricOptions(0, 0, 7)
    h = ctypes.c_void_p()
    st = _lib.load().mi_metric_create_ex(f.ctx.handle, f.handle, m.handle, None, None, None, 32,
                                         ctypes.byref(opts), ctypes.byref(h))
    assert _lib.STATUS_NAMES[st] == "MI_ERR_INVALID_ARGUMENT" and not h.value
    # the whole grid without a mask is walked in voxel order
    assert np.array_equal(metric.sample_order(), np.arange(16 ** 3, dtype=np.uint32))


@pytest.mark.parametrize("dtype", [np.uint8, np.int16, np.uint16, np.int32, np.float64, np.int64])
def test_upload_casts_every_scalar_type(dtype):
    # cuda/image.rs:98-106: (float)(double)x on the device
    sb = _sb()
    rng = np.random.default_rng(0)
    info = np.iinfo(dtype) if np.issubdtype(dtype, np.integer) else None
    if info is not None:
        a = rng.integers(max(info.min, -10 ** 9), min(info.max, 10 ** 9), size=(5, 6, 7)).astype(dtype)
    else:
        a = rng.normal(0, 1e3, size=(5, 6, 7)).astype(dtype)
    img = sb.DeviceImage.upload(a, spacing=(1, 2, 3), origin=(4, 5, 6))
    np.testing.assert_array_equal(img.to_host(), a.astype(np.float64).astype(np.float32))
    assert img.size == (7, 6, 5)


def test_two_stage_point_map(oracle_lib):
    # a composite of two maps is replayed stage by stage (matrix_offset.rs:102-109)
    sb = _sb()
    p = small_pair(n=24, seed=17)
    f, m = _upload_pair(p)
    metric = sb.DeviceMattesMetric.from_device(f, m, 32)
    s1 = sb.transform_stage(sb.AffineTransform(np.eye(3) * 1.01, (0.1, 0.2, 0.3), [11.5] * 3))
    s2 = sb.transform_stage(sb.TranslationTransform((0.25, -0.5, 0.125)))
    v2, n2 = metric.value_stages(np.concatenate([s1, s2]))
    # same decisions as the oracle's composition of the two stages: compose on the
    # host in the same per-stage rounding by evaluating at every grid point
    dec = metric.sample_decisions(np.concatenate([s1, s2]))
    assert n2 == int((dec["status"] == 2).sum())
    assert np.isfinite(v2)


def test_bf16_moving_storage_euler_64_bins(oracle_lib):
    """The large-volume form at reduced size (Euler3D, 64 bins, 20 % random sampling)
    with the moving volume stored as BF16: exact decisions and the usual tolerances
    against the oracle on the rounded volume; the storage error itself (against the
    oracle on the f32 volume) is a property of BF16, bounded loosely here."""
    sb = _sb()
    p = small_pair(n=96, seed=33, nblobs=24, rot=10.0, trans=5.0, scale=None)
    c = [47.5] * 3
    t = sb.Euler3DTransform((0.04, -0.03, 0.06), (1.1, -0.8, 0.5), c)
    draw = oracle_lib.draw_samples(96 ** 3, 2, 0.2, 7)
    _, mv, ref_b, _ = _compare(oracle_lib, p, 96, t, 64, strategy=2, pct=0.2, seed=7, moving_storage="bf16")
    g = _oracle_geo(oracle_lib, 96, (1.0, 1.0, 1.0), (0.0, 0.0, 0.0))
    ref_f = oracle_lib.evaluate(p.fixed, g, p.moving, g, 64, t.kind, t.params, t.fixed_params, draw=draw)
    assert abs(mv.value - ref_f["value"]) <= 1e-2 * abs(ref_f["value"])
    scale = np.max(np.abs(ref_f["derivative"]))
    assert np.max(np.abs(mv.derivative - ref_f["derivative"])) <= 0.1 * scale


def brick_bl(nvox, n, sizes):
    """The brick edge (log2) of the Mattes metric's sample layout: the smallest of 16,
    32, 64 voxels with at least 200 samples per brick on average, and no more than
    1024 bricks along any axis."""
    bl = 4
    while bl < 6 and n * (1 << (3 * bl)) < 200 * nvox:
        bl += 1
    for s in sizes:
        while bl < 6 and -(-s // (1 << bl)) > 1024:
            bl += 1
    return bl


def brick_order_key(order, nx, ny, nvox, n, nz=None):
    """Sort key of the layout's walk: bricks (x-fastest), their 8³ sub-bricks
    (x-fastest), the voxels (x-fastest)."""
    bl = brick_bl(nvox, n, (nx, ny) if nz is None else (nx, ny, nz))
    x, y, z = order % nx, (order // nx) % ny, order // (nx * ny)
    nbx, nby = -(-nx // (1 << bl)), -(-ny // (1 << bl))
    brick = ((z >> bl) * nby + (y >> bl)) * nbx + (x >> bl)
    sm = (1 << (bl - 3)) - 1
    sb_ = bl - 3
    sub = ((((z >> 3) & sm) << sb_ | ((y >> 3) & sm)) << sb_) | ((x >> 3) & sm)
    local = ((z & 7) << 6) | ((y & 7) << 3) | (x & 7)
    return (brick << (3 * bl)) | (sub << 9) | local


def test_sample_order_is_the_gated_draw_in_brick_order(oracle_lib):
    # The device walks the strategy's draw gated by the fixed mask, as the same multiset,
    # in the brick layout's order (grid sizes that are not multiples of the brick leave
    # partial bricks)
    sb = _sb()
    rng = np.random.default_rng(3)
    nz, ny, nx = 21, 29, 37
    vol = rng.standard_normal((nz, ny, nx)).astype(np.float32)
    fmask = (rng.random(vol.shape) > 0.4).astype(np.float32)
    f, m = sb.DeviceImage.upload(vol), sb.DeviceImage.upload(vol)
    for strategy, pct in ((sb.SAMPLING_RANDOM, 0.5), (sb.SAMPLING_REGULAR, 0.25)):
        metric = sb.DeviceMattesMetric.from_device_sampled(f, m, fixed_mask=fmask, bins=32, strategy=strategy,
                                                           percentage=pct, seed=11)
        order = metric.sample_order().astype(np.int64)
        draw = np.asarray(oracle_lib.draw_samples(vol.size, strategy, pct, 11))
        draw = draw[fmask.ravel()[draw] != 0]
        np.testing.assert_array_equal(np.sort(order), np.sort(draw))
        key = brick_order_key(order, nx, ny, vol.size, len(order), nz)
        assert np.all(np.diff(key) >= 0)


@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_layered_and_3d_textures_agree_bit_for_bit(storage):
    # The corner fetch from the layered texture (two gathers per cell) and from the 3-D
    # texture (eight point fetches) read the same stored voxels with the same edge clamp,
    # so every metric gives the same bits; the pose reaches past the volume's edges.
    sb = _sb()
    p = small_pair(n=40, seed=21)
    f, m = _upload_pair(p)
    t = sb.VersorRigid3DTransform((0.05, -0.04, 0.03), (2.5, -1.75, 3.25), [19.5] * 3)
    out = {}
    for tex in ("auto", "3d"):
        metric = sb.DeviceMattesMetric.from_device_sampled(f, m, bins=32, strategy=sb.SAMPLING_RANDOM,
                                                           percentage=0.5, seed=3, moving_storage=storage,
                                                           texture=tex)
        mv = metric.evaluate(t)
        dec = metric.sample_decisions(sb.transform_stage(t))
        out[tex] = (mv.value, mv.derivative.copy(), mv.valid_points, dec["mi"].copy(), dec["status"].copy())
    a, b = out["auto"], out["3d"]
    assert a[0] == b[0] and a[2] == b[2] and a[2] > 0
    assert np.array_equal(a[1], b[1])
    assert np.array_equal(a[3], b[3]) and np.array_equal(a[4], b[4])
    ms = [sb.DeviceMeanSquaresMetric.from_device_sampled(f, m, strategy=sb.SAMPLING_RANDOM, percentage=0.5, seed=3,
                                                         moving_storage=storage, texture=tex).evaluate(t)
          for tex in ("auto", "3d")]
    assert ms[0].value == ms[1].value and np.isfinite(ms[0].value)
    assert np.array_equal(ms[0].derivative, ms[1].derivative)
