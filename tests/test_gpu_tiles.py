"""TMA-staged moving tiles (the histogram pass's other corner source) against the
texture pass: the same decisions and the same corner values, so the same value,
valid count and derivative to the bit, on sampled, whole-grid, masked and BF16-stored
metrics, and through a registration; the evaluation counter shows the staged pass ran.
A moving volume whose x size is not a multiple of four is refused by name."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sb():
    import sitk_b200 as sb
    return sb


def _pair(n, seed):
    from sitk_b200 import synth
    return synth.make_pair(n, 8, seed, 5.0, 3.0, (0.95, 1.05))


def _both(metric, t):
    from sitk_b200.metric import set_tile_staging, get_tile_staging
    set_tile_staging(metric, False)
    a = metric.evaluate(t)
    va = metric.value(t)
    set_tile_staging(metric, True)
    _, n0 = get_tile_staging(metric)
    b = metric.evaluate(t)
    vb = metric.value(t)
    _, n1 = get_tile_staging(metric)
    set_tile_staging(metric, False)
    return a, b, va, vb, n1 - n0


@pytest.mark.parametrize("case", ["random", "full", "masks", "bf16"])
def test_staged_tiles_give_the_texture_bits(case):
    sb = _sb()
    n = 48
    p = _pair(n, 17)
    f, m = sb.DeviceImage.upload(p.fixed), sb.DeviceImage.upload(p.moving)
    kw = dict(bins=32)
    if case == "random":
        kw.update(strategy=sb.SAMPLING_RANDOM, percentage=0.2, seed=5)
    elif case == "masks":
        rng = np.random.default_rng(4)
        kw.update(strategy=sb.SAMPLING_RANDOM, percentage=0.5, seed=5,
                  moving_mask=(rng.random(p.moving.shape) > 0.2).astype(np.uint8),
                  fixed_mask=(rng.random(p.fixed.shape) > 0.3).astype(np.float32))
    elif case == "bf16":
        kw.update(strategy=sb.SAMPLING_RANDOM, percentage=0.2, seed=5, moving_storage="bf16")
    metric = sb.DeviceMattesMetric.from_device_sampled(f, m, **kw)
    # interior bricks are staged, the ones whose cells reach the volume's edge keep the
    # texture: both kinds are present at this pose
    t = sb.VersorRigid3DTransform((0.04, -0.03, 0.05), (1.5, -2.0, 1.0), [(n - 1) / 2.0] * 3)
    a, b, va, vb, ran = _both(metric, t)
    assert ran == 2
    assert a.valid_points == b.valid_points and a.valid_points > 0
    assert a.value == b.value and va == vb == a.value
    assert np.array_equal(a.derivative, b.derivative)


def test_staged_tiles_through_a_registration():
    sb = _sb()
    from sitk_b200 import registration
    from sitk_b200.metric import set_tile_staging, get_tile_staging
    n = 40
    p = _pair(n, 23)
    f, m = sb.DeviceImage.upload(p.fixed), sb.DeviceImage.upload(p.moving)
    out = []
    for on in (False, True):
        metric = sb.DeviceMattesMetric.from_device_sampled(f, m, bins=32, strategy=sb.SAMPLING_RANDOM,
                                                           percentage=0.3, seed=9)
        set_tile_staging(metric, on)
        t = sb.AffineTransform(np.eye(3), (0.0, 0.0, 0.0), [(n - 1) / 2.0] * 3)
        r = registration.register_rsgd(metric, t, iterations=15)
        out.append((t.params.copy(), r.value, r.iterations, get_tile_staging(metric)[1]))
        metric.close()
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1] == out[1][1] and out[0][2] == out[1][2]
    assert out[0][3] == 0 and out[1][3] >= out[1][2]


def test_staged_tiles_refused_for_unaligned_rows():
    sb = _sb()
    from sitk_b200.metric import set_tile_staging
    from sitk_b200._lib import MiError
    rng = np.random.default_rng(1)
    vol = rng.standard_normal((20, 22, 30)).astype(np.float32)  # x size 30
    f, m = sb.DeviceImage.upload(vol), sb.DeviceImage.upload(vol)
    metric = sb.DeviceMattesMetric.from_device_sampled(f, m, bins=16)
    with pytest.raises(MiError) as e:
        set_tile_staging(metric, True)
    assert e.value.name == "MI_ERR_INVALID_ARGUMENT"
