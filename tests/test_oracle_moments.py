"""The oracle's mean-squares and correlation restatements, pinned (CPU only).

The reference holds no golden vectors for either metric; its own pins are
relational (registration/correlation.rs tests: identical images give −1 with a
zero gradient, an affine intensity map of the moving image leaves the value
unchanged, the derivative matches a central finite difference, value() equals
evaluate().value). They are re-created here in 3-D, and both metrics are
cross-checked against an independent numpy FP64 restatement.
"""
import numpy as np
import pytest

AFFINE, EULER3D, VERSOR, TRANSLATION = 0, 1, 2, 3


def _blob(n, c, sigma, amp=100.0, base=10.0):
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    d2 = (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2
    return (base + amp * np.exp(-d2 / (2.0 * sigma * sigma))).astype(np.float32)


def _np_trilinear(vol, c):
    """Linear interpolator value and index-space gradient (transform/interpolator.rs:103-152)
    at continuous indices c (N × 3, x first), clamp-to-edge corners; no inside test."""
    n = np.array(vol.shape[::-1])
    base = np.floor(c).astype(np.int64)
    fr = c - base
    v = np.zeros(len(c))
    g = np.zeros((len(c), 3))
    for corner in range(8):
        bits = [(corner >> d) & 1 for d in range(3)]
        idx = [np.clip(base[:, d] + bits[d], 0, n[d] - 1) for d in range(3)]
        b = vol[idx[2], idx[1], idx[0]].astype(np.float64)
        w = np.ones(len(c))
        for d in range(3):
            w = w * (fr[:, d] if bits[d] else 1.0 - fr[:, d])
        v += w * b
        for j in range(3):
            wj = np.ones(len(c))
            for d in range(3):
                if d != j:
                    wj = wj * (fr[:, d] if bits[d] else 1.0 - fr[:, d])
            g[:, j] += (1.0 if bits[j] else -1.0) * wj * b
    return v, g


def _np_metric(fixed, moving, t, which):
    """Unit spacing, zero origin, identity direction: index = physical. Translation t."""
    n = fixed.shape[0]
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    pts = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1).astype(np.float64)
    c = pts + np.asarray(t, dtype=np.float64)
    inside = np.all((c >= -0.5) & (c < n - 0.5), axis=1)
    c = c[inside]
    f = fixed.ravel()[inside].astype(np.float64)
    mv, g = _np_trilinear(moving, c)
    if which == "ms":
        diff = mv - f
        return np.mean(diff * diff), 2.0 * (diff[:, None] * g).sum(0) / len(diff), int(inside.sum())
    f1 = f - f.mean()
    m1 = mv - mv.mean()
    sff, smm, sfm = (f1 * f1).sum(), (m1 * m1).sum(), (f1 * m1).sum()
    fdm = (f1[:, None] * g).sum(0)
    mdm = (m1[:, None] * g).sum(0)
    value = -sfm * sfm / (sff * smm)
    return value, -2.0 * sfm / (sff * smm) * (fdm - sfm / smm * mdm), int(inside.sum())


@pytest.fixture(scope="module")
def O(oracle_lib):
    return oracle_lib


def _geo(O, n):
    return O.make_geometry((n, n, n))


def test_correlation_identical_images_give_minus_one_and_zero_gradient(O):
    img = _blob(20, (9.5, 10.0, 9.0), 4.0)
    g = _geo(O, 20)
    r = O.correlation(img, g, img, g, TRANSLATION, [0.0, 0.0, 0.0])
    assert abs(r["value"] + 1.0) < 1e-9
    assert np.max(np.abs(r["derivative"])) < 1e-6
    assert r["valid"] == 20 ** 3


def test_correlation_is_invariant_to_an_affine_intensity_map(O):
    fixed = _blob(20, (8.0, 10.0, 9.0), 4.0)
    moving = _blob(20, (11.0, 9.0, 10.0), 4.0)
    rescaled = (2.5 * moving.astype(np.float64) + 7.0).astype(np.float32)
    g = _geo(O, 20)
    t = [1.3, -0.7, 0.4]
    a = O.correlation(fixed, g, moving, g, TRANSLATION, t)["value"]
    b = O.correlation(fixed, g, rescaled, g, TRANSLATION, t)["value"]
    assert abs(a - b) < 1e-6  # the f32 rescale itself rounds the moving voxels


@pytest.mark.parametrize("which", ["ms", "ncc"])
def test_derivative_matches_central_difference(O, which):
    fixed = _blob(20, (10.0, 10.0, 10.0), 4.0)
    moving = _blob(20, (10.0, 10.0, 10.0), 4.0)
    g = _geo(O, 20)
    fn = O.mean_squares if which == "ms" else O.correlation
    p0 = np.array([1.3, -0.7, 0.45])
    an = fn(fixed, g, moving, g, TRANSLATION, p0)["derivative"]
    h = 1e-4
    for k in range(3):
        pp, pm = p0.copy(), p0.copy()
        pp[k] += h
        pm[k] -= h
        fd = (fn(fixed, g, moving, g, TRANSLATION, pp)["value"] - fn(fixed, g, moving, g, TRANSLATION, pm)["value"]) / (2 * h)
        assert abs(fd - an[k]) <= 1e-3 * max(1.0, abs(an[k])), (k, fd, an[k])


@pytest.mark.parametrize("which", ["ms", "ncc"])
def test_value_only_agrees_with_evaluate(O, which):
    fixed = _blob(18, (8.0, 9.0, 9.5), 3.5)
    moving = _blob(18, (9.5, 8.0, 9.0), 3.5)
    g = _geo(O, 18)
    fn = O.mean_squares if which == "ms" else O.correlation
    t = [0.3, -0.6, 0.2]
    a = fn(fixed, g, moving, g, TRANSLATION, t)
    b = fn(fixed, g, moving, g, TRANSLATION, t, derivative=False)
    assert a["valid"] == b["valid"]
    # evaluate scales by 1/count, value() divides: they may differ in the last bit
    assert abs(a["value"] - b["value"]) <= 4e-16 * abs(a["value"])


@pytest.mark.parametrize("which", ["ms", "ncc"])
def test_oracle_matches_independent_numpy_restatement(O, which):
    fixed = _blob(16, (7.0, 8.0, 7.5), 3.0)
    moving = _blob(16, (8.0, 7.0, 8.5), 3.5, amp=80.0)
    g = _geo(O, 16)
    t = [0.37, -0.52, 0.81]
    fn = O.mean_squares if which == "ms" else O.correlation
    r = fn(fixed, g, moving, g, TRANSLATION, t)
    v, d, nv = _np_metric(fixed, moving, t, which)
    assert r["valid"] == nv
    assert abs(r["value"] - v) <= 1e-12 * max(1.0, abs(v))
    assert np.max(np.abs(r["derivative"] - d)) <= 1e-10 * max(1.0, np.max(np.abs(d)))


def test_no_valid_sample_gives_max(O):
    img = _blob(10, (5.0, 5.0, 5.0), 2.0)
    g = _geo(O, 10)
    for fn in (O.mean_squares, O.correlation):
        r = fn(img, g, img, g, TRANSLATION, [100.0, 0.0, 0.0])
        assert r["valid"] == 0 and r["value"] == np.finfo(np.float64).max
        assert np.all(r["derivative"] == 0.0)


def test_constant_moving_is_degenerate_for_correlation_only(O):
    fixed = _blob(10, (5.0, 5.0, 5.0), 2.0)
    flat = np.full((10, 10, 10), 3.0, dtype=np.float32)
    g = _geo(O, 10)
    r = O.correlation(fixed, g, flat, g, TRANSLATION, [0.2, 0.0, 0.0])
    assert r["value"] == np.finfo(np.float64).max and r["valid"] > 0
    m = O.mean_squares(fixed, g, flat, g, TRANSLATION, [0.2, 0.0, 0.0])
    assert m["value"] < np.finfo(np.float64).max
