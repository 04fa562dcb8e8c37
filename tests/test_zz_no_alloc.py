"""The allocation-free value entry point (mi_metric_value_noalloc), through the C ABI.

It exists for callers that may not allocate device memory — an application that runs
the metric inside a device-memory budget it manages itself, or a real-time loop that
must not reach the allocator — and keeps its one scratch buffer in the library's own
device memory. This file is collected last so a run that stops at the first failure has
already run every other test; it passes alone in a fresh process and after the others
(it relies on no state they leave behind).
"""
import ctypes

import numpy as np
import pytest

from conftest import small_pair

pytestmark = pytest.mark.gpu

VALUE_RTOL = 1e-5  # the tolerance the parity tests hold the device value to


def _call(L, ctx, fixed_ptr, f, m, samples, n, info, st, nstage, result):
    return L.mi_metric_value_noalloc(
        ctx.handle, ctypes.c_void_p(fixed_ptr), ctypes.byref(f.geo), ctypes.c_void_p(m.device_ptr()),
        ctypes.byref(m.geo), None if samples is None else ctypes.c_void_p(samples.data_ptr()), n,
        ctypes.byref(info), st.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), nstage,
        ctypes.c_void_p(result.data_ptr()))


def test_noalloc_value_matches_the_metric_object_twice_in_a_row():
    import torch
    import sitk_b200 as sb
    from sitk_b200 import _lib

    L = _lib.load()
    ctx = sb.Context(0)
    p = small_pair(n=40, seed=31, rot=9.0, trans=4.0)
    f = sb.DeviceImage.upload(p.fixed, spacing=(1.0, 1.1, 0.9), origin=(-3.0, 2.0, 1.0), ctx=ctx)
    m = sb.DeviceImage.upload(p.moving, spacing=(1.0, 1.1, 0.9), origin=(-3.0, 2.0, 1.0), ctx=ctx)
    rng = np.random.default_rng(7)
    draw = rng.integers(0, 40 ** 3, size=20000)
    metric = sb.DeviceMattesMetric.from_device_sampled(f, m, samples=draw, bins=50)
    t = sb.AffineTransform(np.eye(3) * 1.01, (0.4, -0.2, 0.3), [-3.0 + 19.5, 2.0 + 1.1 * 19.5, 1.0 + 0.9 * 19.5])
    stage = sb.transform_stage(t)
    expect, expect_valid = metric.value_stages(stage)

    info = _lib.MiMetricInfo()
    _lib.check(L.mi_metric_info_get(metric.handle, ctypes.byref(info)), ctx.handle)
    samples = torch.tensor(draw.astype(np.int64), dtype=torch.int64).to(torch.int32).cuda()
    result = torch.zeros(2, dtype=torch.float64, device="cuda")
    st = np.ascontiguousarray(stage, dtype=np.float64)
    for _ in range(2):
        result.fill_(-1.0)
        torch.cuda.synchronize()
        _lib.check(L.mi_metric_value_noalloc(
            ctx.handle, ctypes.c_void_p(f.device_ptr()), ctypes.byref(f.geo), ctypes.c_void_p(m.device_ptr()),
            ctypes.byref(m.geo), ctypes.c_void_p(samples.data_ptr()), samples.numel(), ctypes.byref(info),
            st.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1, ctypes.c_void_p(result.data_ptr())),
            ctx.handle)
        ctx.sync()
        value, valid = result.cpu().tolist()
        assert int(valid) == expect_valid
        assert abs(value - expect) <= VALUE_RTOL * abs(expect), (value, expect)


def test_noalloc_refuses_more_bins_than_its_scratch_holds():
    import sitk_b200 as sb
    from sitk_b200 import _lib

    L = _lib.load()
    ctx = sb.Context(0)
    p = small_pair(n=16, seed=2)
    f = sb.DeviceImage.upload(p.fixed, ctx=ctx)
    m = sb.DeviceImage.upload(p.moving, ctx=ctx)
    metric = sb.DeviceMattesMetric.from_device(f, m, 100)
    info = _lib.MiMetricInfo()
    _lib.check(L.mi_metric_info_get(metric.handle, ctypes.byref(info)), ctx.handle)
    st = np.ascontiguousarray(sb.transform_stage(sb.TranslationTransform((0.0, 0.0, 0.0))))
    s = L.mi_metric_value_noalloc(ctx.handle, ctypes.c_void_p(f.device_ptr()), ctypes.byref(f.geo),
                                  ctypes.c_void_p(m.device_ptr()), ctypes.byref(m.geo), None, 0,
                                  ctypes.byref(info), st.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1,
                                  ctypes.c_void_p(m.device_ptr()))
    assert _lib.STATUS_NAMES[s] == "MI_ERR_TOO_MANY_HISTOGRAM_BINS"


def test_noalloc_whole_grid_matches_the_metric_object():
    # samples = NULL walks every voxel of the fixed grid, like a metric made with no
    # sampling; two calls in a row give the metric object's value
    import torch
    import sitk_b200 as sb
    from sitk_b200 import _lib

    L = _lib.load()
    ctx = sb.Context(0)
    p = small_pair(n=32, seed=5, rot=7.0, trans=2.0)
    f = sb.DeviceImage.upload(p.fixed, ctx=ctx)
    m = sb.DeviceImage.upload(p.moving, ctx=ctx)
    metric = sb.DeviceMattesMetric.from_device(f, m, 32)
    t = sb.VersorRigid3DTransform((0.01, -0.02, 0.015), (0.4, -0.3, 0.2), [15.5] * 3)
    stage = np.ascontiguousarray(sb.transform_stage(t), dtype=np.float64)
    expect, expect_valid = metric.value_stages(stage)
    info = _lib.MiMetricInfo()
    _lib.check(L.mi_metric_info_get(metric.handle, ctypes.byref(info)), ctx.handle)
    result = torch.zeros(2, dtype=torch.float64, device="cuda")
    for _ in range(2):
        result.fill_(-1.0)
        torch.cuda.synchronize()
        _lib.check(_call(L, ctx, f.device_ptr(), f, m, None, 0, info, stage, 1, result), ctx.handle)
        ctx.sync()
        value, valid = result.cpu().tolist()
        assert int(valid) == expect_valid > 0
        assert abs(value - expect) <= VALUE_RTOL * abs(expect), (value, expect)


def test_noalloc_reports_sample_indices_beyond_the_grid():
    # The sample list is device memory the host cannot check: an index at the voxel
    # count is skipped on the device and reported as value NaN, valid = −(count). The
    # fixed buffer here is larger than the grid its geometry declares, so that index
    # still lies inside the allocation.
    import torch
    import sitk_b200 as sb
    from sitk_b200 import _lib

    L = _lib.load()
    ctx = sb.Context(0)
    n = 24
    p = small_pair(n=n, seed=9)
    f = sb.DeviceImage.upload(p.fixed, ctx=ctx)
    m = sb.DeviceImage.upload(p.moving, ctx=ctx)
    metric = sb.DeviceMattesMetric.from_device(f, m, 32)
    info = _lib.MiMetricInfo()
    _lib.check(L.mi_metric_info_get(metric.handle, ctypes.byref(info)), ctx.handle)
    roomy = torch.zeros(2 * n ** 3, dtype=torch.float32, device="cuda")
    roomy[: n ** 3] = torch.from_numpy(np.ascontiguousarray(p.fixed, dtype=np.float32).ravel()).cuda()
    stage = np.ascontiguousarray(sb.transform_stage(sb.TranslationTransform((0.3, -0.2, 0.1))), dtype=np.float64)
    result = torch.zeros(2, dtype=torch.float64, device="cuda")
    good = torch.tensor([0, 17, 400, n ** 3 - 1], dtype=torch.int32, device="cuda")
    bad = torch.tensor([0, 17, n ** 3, 400, n ** 3 + 5], dtype=torch.int32, device="cuda")
    for samples, want_bad in ((bad, 2), (good, 0), (bad, 2)):
        result.fill_(-1.0)
        torch.cuda.synchronize()
        _lib.check(_call(L, ctx, roomy.data_ptr(), f, m, samples, samples.numel(), info, stage, 1, result),
                   ctx.handle)
        ctx.sync()
        value, valid = result.cpu().tolist()
        if want_bad:
            assert np.isnan(value) and valid == -want_bad
        else:
            assert np.isfinite(value) and 0 < valid <= 4
    # an empty point map, or one longer than the device replays, is refused by name
    for nstage in (0, 9):
        st = np.zeros(12 * max(nstage, 1))
        s = _call(L, ctx, f.device_ptr(), f, m, None, 0, info, st, nstage, result)
        assert _lib.STATUS_NAMES[s] == "MI_ERR_POINT_MAP_STAGE_COUNT"


def test_noalloc_replays_from_a_captured_graph():
    # The documented use under stream capture: one call outside any capture (it looks
    # the scratch array up), then one call captured into a CUDA graph on the context's
    # stream; each replay gives the direct call's value bits.
    import torch
    import sitk_b200 as sb
    from sitk_b200 import _lib

    L = _lib.load()
    ctx = sb.Context(0)
    n = 32
    p = small_pair(n=n, seed=13, rot=6.0, trans=2.0)
    f = sb.DeviceImage.upload(p.fixed, ctx=ctx)
    m = sb.DeviceImage.upload(p.moving, ctx=ctx)
    metric = sb.DeviceMattesMetric.from_device(f, m, 32)
    info = _lib.MiMetricInfo()
    _lib.check(L.mi_metric_info_get(metric.handle, ctypes.byref(info)), ctx.handle)
    t = sb.VersorRigid3DTransform((0.02, 0.01, -0.015), (0.5, 0.2, -0.4), [(n - 1) / 2.0] * 3)
    stage = np.ascontiguousarray(sb.transform_stage(t), dtype=np.float64)
    samples = torch.arange(0, n ** 3, 3, dtype=torch.int32, device="cuda")
    result = torch.zeros(2, dtype=torch.float64, device="cuda")
    _lib.check(_call(L, ctx, f.device_ptr(), f, m, samples, samples.numel(), info, stage, 1, result), ctx.handle)
    ctx.sync()
    direct = result.cpu().tolist()
    assert direct[1] > 0 and np.isfinite(direct[0])

    stream = torch.cuda.ExternalStream(ctx.stream())
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=stream):
        _lib.check(_call(L, ctx, f.device_ptr(), f, m, samples, samples.numel(), info, stage, 1, result),
                   ctx.handle)
    for _ in range(2):
        result.fill_(-1.0)
        torch.cuda.synchronize()
        graph.replay()
        torch.cuda.synchronize()
        assert result.cpu().tolist() == direct
    del graph
