"""Host-side argument handling of DeviceMattesMetric.evaluate (CPU only).

evaluate() reuses ctypes argument buffers across calls and hands them to the C entry
point without ctypes argument conversion. These tests put a stand-in for the C call
behind the same buffers and check that the parameters arrive in place, that the
returned derivative is the caller's own copy (a later call must not change an earlier
result) and that a failing status is raised by name.
"""
import ctypes

import numpy as np
import pytest


def _metric_with_stub(stub):
    from sitk_b200.metric import DeviceMattesMetric
    m = DeviceMattesMetric.__new__(DeviceMattesMetric)
    DeviceMattesMetric.__init__(m, ctypes.c_void_p(None), None)
    m._fn = stub(m)
    return m


def test_parameters_arrive_and_results_are_independent_copies():
    import sitk_b200 as sb
    seen = []

    def stub(m):
        def call(handle, kind, p, n, fp, nf, vref, d, nref):
            seen.append((kind, list(p[:n]), None if fp is None else list(fp[:nf])))
            for i in range(n):
                d[i] = 10.0 * len(seen) + i
            m._v.value = -0.5 * len(seen)
            m._n.value = 1000 + len(seen)
            return 0
        return call

    m = _metric_with_stub(stub)
    t = sb.VersorRigid3DTransform((0.05, -0.04, 0.03), (2.5, -1.75, 3.25), [1.0, 2.0, 3.0])
    r1 = m.evaluate(t)
    t2 = sb.TranslationTransform((0.25, -0.5, 0.125))
    r2 = m.evaluate(t2)
    assert seen[0] == (t.kind, list(t.params), list(t.fixed_params))
    assert seen[1] == (t2.kind, list(t2.params), None)
    assert r1.value == -0.5 and r1.valid_points == 1001
    np.testing.assert_array_equal(r1.derivative, 10.0 + np.arange(6))
    np.testing.assert_array_equal(r2.derivative, 20.0 + np.arange(3))
    # the first result is not a view of the reused buffer
    np.testing.assert_array_equal(r1.derivative, 10.0 + np.arange(6))


def test_failing_status_is_raised_by_name():
    import sitk_b200 as sb
    from sitk_b200 import _lib

    def stub(m):
        return lambda *a: 1  # MI_ERR_INVALID_ARGUMENT

    m = _metric_with_stub(stub)
    m.ctx = type("Ctx", (), {"handle": None})()
    with pytest.raises(_lib.MiError) as e:
        m.evaluate(sb.TranslationTransform((0.0, 0.0, 0.0)))
    assert e.value.name == "MI_ERR_INVALID_ARGUMENT"
