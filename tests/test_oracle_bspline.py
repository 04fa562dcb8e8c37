"""The oracle's B-spline transform and sparse-support Mattes path, pinned (CPU only).

Re-creates in 3-D the reference's own pins (transform/bspline.rs tests: zero
coefficients are the identity, a constant coefficient field is a uniform translation,
a single coefficient displaces by the hand-derived weight and nothing outside its
support, points outside the valid region are unmapped; registration/mattes.rs:952-1010:
the derivative matches a central finite difference) and cross-checks the transform
against an independent numpy restatement.
"""
import numpy as np
import pytest


def _geo(O, n, spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0)):
    return O.make_geometry((n, n, n), spacing, origin)


def _transform(n, mesh, spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0)):
    from sitk_b200.transforms import BSplineTransform
    from sitk_b200.metric import geometry
    return BSplineTransform.from_image_domain(geometry((n, n, n), spacing, origin), mesh)


def _np_b3(u):
    a = np.abs(u)
    return np.where(a < 1.0, (4.0 - 6.0 * a * a + 3.0 * a ** 3) / 6.0,
                    np.where(a < 2.0, (2.0 - a) ** 3 / 6.0, 0.0))


def _np_point(t, x):
    """Independent restatement: grid index, valid-region test, 4³ weights."""
    fp = t.fixed_params
    size = fp[0:3].astype(int)
    org, sp, d = fp[3:6], fp[6:9], fp[9:18].reshape(3, 3)
    idx = np.linalg.solve(d @ np.diag(sp), np.asarray(x, dtype=np.float64) - org)
    if np.any(idx < 1.0) or np.any(idx >= size - 2.0):
        return np.array(x, dtype=np.float64)
    start = np.floor(idx - 1.0).astype(int)
    n = size[0] * size[1] * size[2]
    c = t.params.reshape(3, size[2], size[1], size[0])
    disp = np.zeros(3)
    for kz in range(4):
        for ky in range(4):
            for kx in range(4):
                g = np.array([start[0] + kx, start[1] + ky, start[2] + kz])
                w = np.prod(_np_b3(idx - g))
                disp += w * c[:, g[2], g[1], g[0]]
    return np.asarray(x, dtype=np.float64) + disp


def test_zero_coefficients_are_the_identity(oracle_lib):
    t = _transform(20, (4, 4, 4))
    for x in ([3.2, 7.7, 11.1], [0.0, 0.0, 0.0], [19.0, 5.5, 2.25]):
        assert np.array_equal(oracle_lib.bspline_transform_point(t.fixed_params, t.params, x), x)


def test_constant_field_is_a_uniform_translation(oracle_lib):
    t = _transform(20, (3, 4, 5))
    n = t.nparams // 3
    p = np.concatenate([np.full(n, 1.5), np.full(n, -0.75), np.full(n, 0.25)])
    t.set_parameters(p)
    for x in ([3.2, 7.7, 11.1], [10.0, 10.0, 10.0], [15.9, 2.4, 8.8]):
        y = oracle_lib.bspline_transform_point(t.fixed_params, t.params, x)
        np.testing.assert_allclose(y - np.asarray(x), [1.5, -0.75, 0.25], rtol=0, atol=1e-12)


def test_single_coefficient_displaces_by_its_weight_and_only_inside_its_support(oracle_lib):
    t = _transform(16, (4, 4, 4))
    gs = t.grid_size
    n = gs[0] * gs[1] * gs[2]
    cp = (3, 2, 3)  # control point (x, y, z); the valid region is [1, 5) per axis
    flat = cp[0] + gs[0] * (cp[1] + gs[1] * cp[2])
    p = np.zeros(3 * n)
    p[1 * n + flat] = 2.0  # y coefficient
    t.set_parameters(p)
    fp = t.fixed_params
    org, sp = fp[3:6], fp[6:9]
    # a point whose grid index is cp + (0.3, −0.6, 0.8): weight Π B₃(idx − cp)
    idx = np.array(cp, dtype=np.float64) + np.array([0.3, -0.6, 0.8])
    x = org + sp * idx
    y = oracle_lib.bspline_transform_point(fp, p, x)
    w = np.prod(_np_b3(np.array([0.3, -0.6, 0.8])))
    np.testing.assert_allclose(y - x, [0.0, 2.0 * w, 0.0], rtol=0, atol=1e-12)
    # outside the 4³ support: untouched
    far = org + sp * (np.array(cp, dtype=np.float64) + np.array([-2.0, 0.1, 0.0]))
    assert np.array_equal(oracle_lib.bspline_transform_point(fp, p, far), far)


def test_points_outside_the_valid_region_are_unmapped(oracle_lib):
    t = _transform(16, (4, 4, 4))
    t.set_parameters(np.linspace(-1.0, 1.0, t.nparams))
    fp = t.fixed_params
    org, sp = fp[3:6], fp[6:9]
    x = org + sp * np.array([0.5, 3.0, 3.0])  # grid index below the valid lower limit 1
    assert np.array_equal(oracle_lib.bspline_transform_point(fp, t.params, x), x)


def test_transform_matches_the_numpy_restatement(oracle_lib):
    rng = np.random.default_rng(9)
    t = _transform(24, (3, 5, 4), spacing=(1.1, 0.9, 1.2), origin=(-3.0, 2.0, 1.0))
    t.set_parameters(0.4 * rng.standard_normal(t.nparams))
    for _ in range(200):
        x = np.array([-3.0, 2.0, 1.0]) + rng.uniform(0, 24, size=3) * np.array([1.1, 0.9, 1.2])
        np.testing.assert_allclose(oracle_lib.bspline_transform_point(t.fixed_params, t.params, x),
                                   _np_point(t, x), rtol=0, atol=1e-12)


def _pair(n):
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    c = (n - 1) / 2.0
    d2 = (x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2
    fixed = np.exp(-d2 / (2.0 * (n / 4.0) ** 2)).astype(np.float32)
    moving = (1.0 - np.exp(-((x - c - 0.7) ** 2 + (y - c) ** 2 + (z - c + 0.4) ** 2) / (2.0 * (n / 4.0) ** 2))
              ).astype(np.float32)
    return fixed, moving


def test_bspline_mattes_derivative_matches_central_difference(oracle_lib):
    n = 18
    fixed, moving = _pair(n)
    g = _geo(oracle_lib, n)
    t = _transform(n, (3, 3, 3))
    p0 = np.array([((i * 31 % 13) - 6.0) * 0.05 for i in range(t.nparams)])
    r = oracle_lib.bspline_mattes(fixed, g, moving, g, 32, t.fixed_params, p0)
    an = r["derivative"]
    h = 1e-3
    checked = 0
    for k in np.argsort(-np.abs(an))[:12]:
        pp, pm = p0.copy(), p0.copy()
        pp[k] += h
        pm[k] -= h
        fd = (oracle_lib.bspline_mattes(fixed, g, moving, g, 32, t.fixed_params, pp, derivative=False)["value"] -
              oracle_lib.bspline_mattes(fixed, g, moving, g, 32, t.fixed_params, pm, derivative=False)["value"]) / (2 * h)
        assert abs(fd - an[k]) < 5e-3 * max(1.0, abs(an[k])), (k, fd, an[k])
        checked += 1
    assert checked >= 10


def test_zero_field_equals_the_identity_affine_value(oracle_lib):
    # a zero coefficient field maps every point to itself, so the value is the
    # global-support metric's at the identity affine
    n = 16
    fixed, moving = _pair(n)
    g = _geo(oracle_lib, n)
    t = _transform(n, (2, 2, 2))
    b = oracle_lib.bspline_mattes(fixed, g, moving, g, 32, t.fixed_params, t.params)
    a = oracle_lib.evaluate(fixed, g, moving, g, 32, 3, [0.0, 0.0, 0.0])
    assert b["valid"] == a["valid"]
    assert b["value"] == a["value"]
