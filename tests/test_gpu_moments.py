"""Mean squares and correlation on the device vs the oracle, through the C ABI.

Contract (the reference's own device pins, tests/cuda_mean_squares.rs:97-182 and
tests/cuda_correlation.rs): the valid-sample count equals the oracle's exactly; value
and every derivative component agree within 1e-9 in the reference's measure
|gpu − cpu| / (1 + |cpu|) (reduction rounding only); results are bit-identical run
to run.
"""
import numpy as np
import pytest

from conftest import small_pair

pytestmark = pytest.mark.gpu

BAND = 1e-9


def _rel(g, c):
    return np.abs(np.asarray(g) - np.asarray(c)) / (1.0 + np.abs(np.asarray(c)))


def _check(oracle, p, n, transform, which, spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0), strategy=None,
           pct=1.0, seed=0, fmask=None, mmask=None):
    import sitk_b200 as sb
    f = sb.DeviceImage.upload(p.fixed, spacing, origin)
    m = sb.DeviceImage.upload(p.moving, spacing, origin)
    cls = sb.DeviceMeanSquaresMetric if which == "ms" else sb.DeviceCorrelationMetric
    metric = cls.from_device_sampled(f, m, fixed_mask=fmask, moving_mask=mmask, strategy=strategy,
                                     percentage=pct, seed=seed)
    draw = oracle.draw_samples(n ** 3, strategy, pct, seed) if strategy else None
    g = oracle.make_geometry((n, n, n), spacing, origin)
    fn = oracle.mean_squares if which == "ms" else oracle.correlation
    ref = fn(p.fixed, g, p.moving, g, transform.kind, transform.params, transform.fixed_params, fmask=fmask,
             mmask=mmask, draw=draw)
    mv = metric.evaluate(transform)
    assert mv.valid_points == ref["valid"] > 0
    assert _rel(mv.value, ref["value"]) <= BAND, (mv.value, ref["value"])
    assert np.max(_rel(mv.derivative, ref["derivative"])) <= BAND, (mv.derivative, ref["derivative"])
    assert np.any(np.abs(ref["derivative"]) > 1e-6)
    # the value-only path walks the same samples
    refv = fn(p.fixed, g, p.moving, g, transform.kind, transform.params, transform.fixed_params, fmask=fmask,
              mmask=mmask, draw=draw, derivative=False)
    assert _rel(metric.value(transform), refv["value"]) <= BAND
    # bit-identical run to run
    again = metric.evaluate(transform)
    assert again.value == mv.value and np.array_equal(again.derivative, mv.derivative)
    metric.close()
    f.free()
    m.free()
    return mv, ref


@pytest.mark.parametrize("which", ["ms", "ncc"])
def test_euler_full_grid(oracle_lib, which):
    import sitk_b200 as sb
    p = small_pair(n=40, seed=3)
    t = sb.Euler3DTransform((0.06, -0.04, 0.03), (2.5, -1.5, 0.75), [20.0] * 3)
    _check(oracle_lib, p, 40, t, which)


@pytest.mark.parametrize("which", ["ms", "ncc"])
def test_affine_random_sampling_nonunit_geometry(oracle_lib, which):
    import sitk_b200 as sb
    p = small_pair(n=44, seed=8, rot=9.0, trans=4.0)
    sp, org = (1.1, 0.9, 1.3), (-5.0, 3.0, 1.5)
    c = [org[d] + sp[d] * 21.5 for d in range(3)]
    A = np.eye(3) + 0.02 * np.array([[1, -1, 0.5], [0.3, -0.5, 1], [0.2, 0.1, -1]])
    t = sb.AffineTransform(A, (0.6, -0.9, 0.4), c)
    _check(oracle_lib, p, 44, t, which, spacing=sp, origin=org, strategy=2, pct=0.25, seed=99)


@pytest.mark.parametrize("which", ["ms", "ncc"])
def test_versor_with_both_masks(oracle_lib, which):
    import sitk_b200 as sb
    p = small_pair(n=36, seed=12, rot=8.0, trans=3.0, scale=None)
    rng = np.random.default_rng(4)
    fmask = (rng.random((36, 36, 36)) > 0.3).astype(np.uint8)
    mmask = (rng.random((36, 36, 36)) > 0.2).astype(np.uint8)
    t = sb.VersorRigid3DTransform((0.02, -0.01, 0.03), (0.4, -0.7, 0.5), [17.5] * 3)
    _check(oracle_lib, p, 36, t, which, fmask=fmask, mmask=mmask)


def test_samples_on_cell_walls_take_the_reference_cell(oracle_lib):
    """An integer translation puts every sample on a moving-grid cell wall, where the
    interpolant's gradient jumps; the device must take the reference's side."""
    import sitk_b200 as sb
    p = small_pair(n=32, seed=5)
    t = sb.TranslationTransform((1.0, -2.0, 0.0))
    for which in ("ms", "ncc"):
        _check(oracle_lib, p, 32, t, which)


def test_degenerate_cases_give_max():
    import sitk_b200 as sb
    p = small_pair(n=24, seed=2)
    f = sb.DeviceImage.upload(p.fixed)
    m = sb.DeviceImage.upload(p.moving)
    flat = sb.DeviceImage.upload(np.full((24, 24, 24), 7.0, dtype=np.float32))
    far = sb.TranslationTransform((500.0, 0.0, 0.0))
    for cls in (sb.DeviceMeanSquaresMetric, sb.DeviceCorrelationMetric):
        metric = cls.from_device(f, m)
        r = metric.evaluate(far)
        assert r.valid_points == 0 and r.value == np.finfo(np.float64).max and np.all(r.derivative == 0)
        metric.close()
    ncc = sb.DeviceCorrelationMetric.from_device(f, flat)
    r = ncc.evaluate(sb.TranslationTransform((0.3, 0.0, 0.0)))
    assert r.valid_points > 0 and r.value == np.finfo(np.float64).max
    ncc.close()
    # a constant image is not refused by these metrics (the Mattes metric refuses it)
    ms = sb.DeviceMeanSquaresMetric.from_device(f, flat)
    assert ms.evaluate(sb.TranslationTransform((0.3, 0.0, 0.0))).value < np.finfo(np.float64).max
    ms.close()
