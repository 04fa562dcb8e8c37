"""The allocation-free value entry point (mi_metric_value_noalloc), through the C ABI.

It exists for callers that may not allocate device memory — code running under CUDA
graph capture, hosts with a fixed memory budget, real-time loops — and keeps its one
scratch buffer in the library's own device memory. This file is collected last so a
run that stops at the first failure has already run every other test; it passes alone
in a fresh process and after the others (it relies on no state they leave behind).
"""
import ctypes

import numpy as np
import pytest

from conftest import small_pair

pytestmark = pytest.mark.gpu

VALUE_RTOL = 1e-5  # the tolerance the parity tests hold the device value to


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
