"""Kernels' dynamic shared-memory limits are raised per launch shape and never lowered:
a metric with many bins (a histogram pass above the default 48 KB of shared memory)
keeps evaluating after a metric with few bins is created, and gives the same bits as
before it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_a_later_metric_with_fewer_bins_keeps_the_larger_limit():
    import sitk_b200 as sb
    from sitk_b200 import synth
    n = 40
    p = synth.make_pair(n, 8, 23, 5.0, 3.0, (0.95, 1.05))
    f, m = sb.DeviceImage.upload(p.fixed), sb.DeviceImage.upload(p.moving)
    t = sb.VersorRigid3DTransform((0.03, -0.02, 0.04), (1.0, -1.5, 0.5), [(n - 1) / 2.0] * 3)
    big = sb.DeviceMattesMetric.from_device_sampled(f, m, bins=64, strategy=sb.SAMPLING_RANDOM,
                                                    percentage=0.3, seed=3)
    before = big.evaluate(t)
    small = sb.DeviceMattesMetric.from_device_sampled(f, m, bins=8, strategy=sb.SAMPLING_RANDOM,
                                                      percentage=0.3, seed=3)
    s = small.evaluate(t)
    after = big.evaluate(t)
    assert s.valid_points > 0
    assert after.valid_points == before.valid_points > 0
    assert after.value == before.value
    assert np.array_equal(after.derivative, before.derivative)
    small.close()
    big.close()
