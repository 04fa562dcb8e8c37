"""Multi-resolution pyramid level: recursive Gaussian smoothing, shrink geometry and
linear resampling onto the coarse grid (registration/method.rs:2416 prepare_level).

The reference holds its device pyramid to the host filters bit for bit
(cuda/ops/pyramid.rs, pyramid_parity.rs); the device kernels here are held to the
oracle's serial FP64 restatement the same way. The oracle itself is pinned to the
reference's own filter tests (filters/recursive_gaussian.rs tests): constants
preserved, unit impulse mass, symmetry, the 0.938·σ² impulse variance of the
Farnebäck zero-order coefficients, physical sigma scaling with spacing.
"""
import numpy as np
import pytest


def _geo(oracle, size, spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0), direction=None):
    g = oracle.make_geometry(size, spacing=spacing, origin=origin)
    if direction is not None:
        for i in range(9):
            g.direction[i] = direction[i]
    return g


def test_oracle_gaussian_preserves_a_constant(oracle_lib):
    # recursive_gaussian.rs tests: constant_image_is_preserved
    g = _geo(oracle_lib, (16, 12, 10))
    v = np.full((10, 12, 16), 5.0, dtype=np.float32)
    out = oracle_lib.recursive_gaussian(v, g, (2.0, 1.5, 3.0))
    assert np.max(np.abs(out - 5.0)) < 1e-5


def test_oracle_gaussian_zero_sigma_is_identity(oracle_lib):
    g = _geo(oracle_lib, (9, 8, 7))
    v = np.random.default_rng(1).random((7, 8, 9)).astype(np.float32)
    np.testing.assert_array_equal(oracle_lib.recursive_gaussian(v, g, (0.0, 0.0, 0.0)), v)


def test_oracle_gaussian_impulse_width_is_the_farneback_fraction_of_sigma(oracle_lib):
    # recursive_gaussian.rs tests: impulse_response_width_matches_the_itk_recursive_gaussian
    n, c, sigma = 201, 100, 4.0
    g = _geo(oracle_lib, (n, 1, 1))
    v = np.zeros((1, 1, n), dtype=np.float32)
    v[0, 0, c] = 1.0
    out = oracle_lib.recursive_gaussian(v, g, (sigma, 0.0, 0.0)).astype(np.float64).ravel()
    assert abs(out.sum() - 1.0) < 1e-6  # the reference's 1e-7 band, widened for the f32 result
    ratio = np.sum(out * (np.arange(n) - c) ** 2) / sigma ** 2
    assert 0.935 <= ratio <= 0.941


def test_oracle_gaussian_impulse_conserves_mass_and_is_symmetric(oracle_lib):
    # recursive_gaussian.rs tests: interior_impulse_conserves_mass_and_is_symmetric (in 3-D)
    n, c = 41, 20
    g = _geo(oracle_lib, (n, n, n))
    v = np.zeros((n, n, n), dtype=np.float32)
    v[c, c, c] = 100.0
    out = oracle_lib.recursive_gaussian(v, g, (2.0, 2.0, 2.0)).astype(np.float64)
    assert abs(out.sum() - 100.0) < 1e-3
    assert 0.0 < out[c, c, c] < 100.0
    for a, b in ((out[c, c, c - 1], out[c, c, c + 1]), (out[c, c - 1, c], out[c, c + 1, c]),
                 (out[c - 1, c, c], out[c + 1, c, c])):
        assert abs(a - b) < 1e-6


def test_oracle_physical_sigma_accounts_for_spacing(oracle_lib):
    n = 21
    v = np.zeros((n, n, n), dtype=np.float32)
    v[10, 10, 10] = 100.0
    fine = oracle_lib.recursive_gaussian(v, _geo(oracle_lib, (n, n, n), (1.0, 1.0, 1.0)), (2.0, 2.0, 2.0))
    coarse = oracle_lib.recursive_gaussian(v, _geo(oracle_lib, (n, n, n), (2.0, 2.0, 2.0)), (2.0, 2.0, 2.0))
    assert coarse[10, 10, 10] > fine[10, 10, 10]


def test_oracle_resample_onto_its_own_grid_is_the_identity(oracle_lib):
    g = _geo(oracle_lib, (11, 9, 7), (0.7, 1.3, 2.0), (-4.0, 3.0, 1.5))
    v = np.random.default_rng(3).random((7, 9, 11)).astype(np.float32)
    np.testing.assert_array_equal(oracle_lib.resample_linear(v, g, g), v)


SHRINK_CASES = [
    ((256, 256, 256), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0), None, (4, 4, 4)),
    ((63, 50, 17), (0.8, 0.9, 1.1), (-3.0, 2.0, 1.0), None, (2, 3, 4)),
    ((10, 3, 5), (1.5, 1.0, 2.5), (4.0, -1.0, 0.5), None, (4, 4, 8)),
    ((40, 36, 44), (1.0, 1.2, 0.9), (1.0, 2.0, 3.0), (0.0, -1.0, 0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0), (3, 2, 5)),
]


@pytest.mark.parametrize("case", SHRINK_CASES)
def test_shrink_geometry_matches_the_oracle(oracle_lib, case):
    from sitk_b200 import metric
    size, sp, org, direction, f = case
    og = _geo(oracle_lib, size, sp, org, direction)
    lg = metric.geometry(size, sp, org, direction or (1, 0, 0, 0, 1, 0, 0, 0, 1))
    o = oracle_lib.shrink_geometry(og, f)
    d = metric.shrink_geometry(lg, f)
    for i in range(3):
        assert d.size[i] == o.size[i]
        assert d.spacing[i] == o.spacing[i]
        assert d.origin[i] == o.origin[i]
    for i in range(9):
        assert d.direction[i] == o.direction[i]


def _blob_volume(size, seed):
    rng = np.random.default_rng(seed)
    nx, ny, nz = size
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    v = np.zeros((nz, ny, nx))
    for _ in range(6):
        c = rng.uniform(0, 1, 3) * np.array([nx, ny, nz])
        s = rng.uniform(2, 6)
        v += rng.uniform(50, 200) * np.exp(-((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) / (2 * s * s))
    v += rng.normal(0, 3, v.shape)
    return v.astype(np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("sigma", [(2.0, 1.5, 0.0), (1.0, 1.0, 1.0), (0.0, 3.2, 0.7)])
def test_device_smoothing_is_the_oracle_bit_for_bit(oracle_lib, sigma):
    import sitk_b200 as sb
    size, sp, org = (40, 36, 44), (1.0, 1.2, 0.9), (1.0, 2.0, 3.0)
    v = _blob_volume(size, 5)
    d = sb.DeviceImage.upload(v, sp, org).smooth(sigma).to_host()
    o = oracle_lib.recursive_gaussian(v, _geo(oracle_lib, size, sp, org), sigma)
    np.testing.assert_array_equal(d, o)


@pytest.mark.gpu
def test_device_smoothing_refuses_a_short_axis():
    import sitk_b200 as sb
    from sitk_b200._lib import MiError
    img = sb.DeviceImage.upload(np.ones((3, 8, 8), dtype=np.float32))
    with pytest.raises(MiError):
        img.smooth((1.0, 1.0, 1.0))
    img.smooth((1.0, 1.0, 0.0))  # a short axis that is not smoothed is fine


@pytest.mark.gpu
@pytest.mark.parametrize("case", SHRINK_CASES[1:])
def test_device_resample_onto_the_shrunk_grid_is_the_oracle_bit_for_bit(oracle_lib, case):
    import sitk_b200 as sb
    from sitk_b200 import metric
    size, sp, org, direction, f = case
    v = _blob_volume(size, 9)
    img = sb.DeviceImage.upload(v, sp, org, direction or (1, 0, 0, 0, 1, 0, 0, 0, 1))
    grid = metric.shrink_geometry(img.geo, f)
    d = img.resample(grid, fill=-7.0).to_host()
    og = _geo(oracle_lib, size, sp, org, direction)
    o = oracle_lib.resample_linear(v, og, oracle_lib.shrink_geometry(og, f), -7.0)
    np.testing.assert_array_equal(d, o)


@pytest.mark.gpu
def test_device_pyramid_levels_are_the_oracle_bit_for_bit(oracle_lib):
    # the 256³ rigid schedule (shrink 4/2/1, sigma 2/1/0) on a smaller volume
    import sitk_b200 as sb
    from sitk_b200 import metric
    n = 48
    fixed, moving = _blob_volume((n, n, n), 11), _blob_volume((n, n, n), 12)
    f = sb.DeviceImage.upload(fixed)
    m = sb.DeviceImage.upload(moving)
    g = _geo(oracle_lib, (n, n, n))
    for factor, sigma in ((4, 2.0), (2, 1.0), (1, 0.0)):
        fl, ml = metric.pyramid_level(f, m, sigma, factor)
        ofl, ogeo, oml = oracle_lib.pyramid_level(fixed, g, moving, g, sigma, (factor,) * 3)
        assert fl.size == tuple(int(ogeo.size[i]) for i in range(3))
        for i in range(3):
            assert fl.geo.origin[i] == ogeo.origin[i] and fl.geo.spacing[i] == ogeo.spacing[i]
        np.testing.assert_array_equal(fl.to_host(), ofl)
        np.testing.assert_array_equal(ml.to_host(), oml)


@pytest.mark.gpu
def test_nearest_resample_matches_the_oracle_bitwise(oracle_lib):
    """transform/interpolator.rs:36-54 through the identity (the level-mask resample of
    registration/method.rs:3068-3110), on a shrunk grid of a non-unit geometry."""
    import sitk_b200 as sb
    from sitk_b200.metric import shrink_geometry
    import oracle
    rng = np.random.default_rng(2)
    vol = (rng.random((30, 26, 22)) * 100).astype(np.float32)
    sp, org = (0.9, 1.2, 1.05), (-4.0, 3.0, 1.5)
    img = sb.DeviceImage.upload(vol, sp, org)
    for factors in ((2, 2, 2), (3, 1, 2), (1, 1, 1)):
        grid = shrink_geometry(img.geo, factors)
        out = img.resample_nearest(grid, 0.0).to_host()
        gi = oracle.make_geometry((22, 26, 30), sp, org)
        go = oracle.shrink_geometry(gi, factors)
        ref = oracle.resample_nearest(vol, gi, go, 0.0)
        assert out.shape == ref.shape
        assert np.array_equal(out.view(np.uint32), ref.view(np.uint32)), factors
