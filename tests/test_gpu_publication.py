"""The split form hands its result to the host through mapped memory: the last kernel
writes value, valid count, derivative and error word, then a tag hashing them with the
evaluation's sequence number, and the host takes the result once the tag matches what
it reads. Calls that wait on the stream instead (timing enabled) are the reference:
value-only and value+derivative calls interleaved many times give their bits every
time, so no call takes a previous call's tag or a partly arrived result."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_polled_results_match_stream_synchronised_ones():
    import sitk_b200 as sb
    from sitk_b200 import synth
    from sitk_b200.metric import enable_timing
    n = 48
    p = synth.make_pair(n, 8, 29, 5.0, 3.0, (0.95, 1.05))
    f, m = sb.DeviceImage.upload(p.fixed), sb.DeviceImage.upload(p.moving)
    metric = sb.DeviceMattesMetric.from_device_sampled(f, m, bins=32, strategy=sb.SAMPLING_RANDOM,
                                                       percentage=0.25, seed=11)
    poses = [sb.VersorRigid3DTransform((0.01 * k, -0.02, 0.015 * k), (0.3 * k, -0.5, 0.2), [(n - 1) / 2.0] * 3)
             for k in range(3)]
    enable_timing(metric, True)
    ref = [(metric.evaluate(t), metric.value(t)) for t in poses]
    enable_timing(metric, False)
    for it in range(40):
        k = it % 3
        r = metric.evaluate(poses[k])
        v = metric.value(poses[k])
        want, want_v = ref[k]
        assert r.value == want.value and r.valid_points == want.valid_points
        assert np.array_equal(r.derivative, want.derivative)
        assert v == want_v == want.value
    metric.close()
