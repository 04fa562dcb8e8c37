"""CPU tests that pin the oracle (no GPU).

The reference (Rust) cannot run here and holds no golden vectors for this metric,
so the oracle is pinned by (1) published SplitMix64 vectors, (2) re-creations of the
reference's own relational tests (file:line cited per test), and (3) agreement with
the independent numpy oracle on every per-sample decision and on the value.
"""
import math

import numpy as np
import pytest

from conftest import geo_dict, small_pair

import np_oracle


def _geo(oracle, size, **kw):
    return oracle.make_geometry(size, **kw)


# --- (1) published vectors -------------------------------------------------------

def test_splitmix64_matches_published_vectors(oracle_lib):
    # Vigna's splitmix64.c reference outputs for seed 1234567, and the well-known
    # first output for seed 0 (0xE220A8397B1DCDAF).
    assert oracle_lib.splitmix64(1234567, 5) == [
        6457827717110365317, 3203168211198807973, 9817491932198370423,
        4593380528125082431, 16408922859458223821]
    assert oracle_lib.splitmix64(0, 1) == [0xE220A8397B1DCDAF]


def test_draw_samples_semantics(oracle_lib):
    # metric.rs:419-437: Random = floor(N·pct) draws with replacement, next_u64 % N.
    d = oracle_lib.draw_samples(1000, 2, 0.1, 42)
    assert d.size == 100
    raw = oracle_lib.splitmix64(42, 100)
    assert d.tolist() == [r % 1000 for r in raw]
    # Regular = every ceil(1/pct)-th voxel.
    r = oracle_lib.draw_samples(10, 1, 0.3, 0)
    assert r.tolist() == [0, 4, 8]
    assert oracle_lib.draw_samples(10, 0, 1.0, 0) is None


# --- (2) relational pins re-created from the reference's tests -----------------

def test_round_half_integer_up(oracle_lib):
    # core/coord.rs:185-191 and its tests: half toward +inf.
    f = oracle_lib.round_half_integer_up
    assert [f(1.5), f(2.5), f(-1.5), f(-0.5), f(0.4999999999999999)] == [2, 3, -1, 0, 0]


def test_cubic_bspline_partition_of_unity(oracle_lib):
    # mattes.rs:821 — the four taps of any fractional position sum to 1.
    rng = np.random.default_rng(1)
    for t in rng.uniform(0, 1, 50):
        u = np.array([-1 - t, -t, 1 - t, 2 - t])
        v, _ = oracle_lib.cubic_bspline(u)
        assert abs(v.sum() - 1.0) < 1e-14


def test_cubic_bspline_derivative_matches_fd(oracle_lib):
    # mattes.rs:833
    u = np.linspace(-1.95, 1.95, 79)
    h = 1e-6
    v1, _ = oracle_lib.cubic_bspline(u + h)
    v0, _ = oracle_lib.cubic_bspline(u - h)
    _, d = oracle_lib.cubic_bspline(u)
    assert np.max(np.abs((v1 - v0) / (2 * h) - d)) < 1e-6


def test_kahan_sum_recovers_what_naive_drops(oracle_lib):
    # core/compensated.rs:213-226 (the pin mattes.rs:856 relies on): 1e17 then a
    # thousand 1.0s — the naive walk provably loses them, the compensated one does not.
    terms = np.array([1.0e17] + [1.0] * 1000)
    naive = 0.0
    for t in terms:
        naive += t
    assert naive != 1.0e17 + 1000.0
    assert oracle_lib.kahan_sum(terms) == 1.0e17 + 1000.0


def test_kahan_keeps_itks_blind_spot(oracle_lib):
    # core/compensated.rs:237-250: [1, 1e100, 1, −1e100] sums to 0.0 (not Neumaier's 2.0).
    assert oracle_lib.kahan_sum(np.array([1.0, 1.0e100, 1.0, -1.0e100])) == 0.0


def test_refusals(oracle_lib):
    # mattes.rs:906 (constant image) and :920 (too few bins)
    p = small_pair()
    g = _geo(oracle_lib, (20, 20, 20))
    with pytest.raises(oracle_lib.OracleError) as e:
        oracle_lib.evaluate(p.fixed, g, p.moving, g, 4, 0, np.eye(3).ravel().tolist() + [0, 0, 0])
    assert e.value.code == 1
    with pytest.raises(oracle_lib.OracleError) as e:
        oracle_lib.evaluate(np.full_like(p.fixed, 3.0), g, p.moving, g, 50, 0,
                            np.eye(3).ravel().tolist() + [0, 0, 0])
    assert e.value.code == 2


def test_mi_is_minimised_at_alignment(oracle_lib):
    # mattes.rs:931 — value (−MI) is lowest at the true alignment.
    from sitk_b200 import synth
    rng = np.random.Generator(np.random.PCG64(3))
    vol = synth.blob_phantom(24, 6, rng).astype(np.float32)
    g = _geo(oracle_lib, (24, 24, 24))
    vals = []
    for tx in (-2.0, -1.0, 0.0, 1.0, 2.0):
        r = oracle_lib.evaluate(vol, g, vol, g, 32, 3, [tx, 0.0, 0.0], derivative=False)
        vals.append(r["value"])
    assert np.argmin(vals) == 2


def test_derivative_matches_central_difference(oracle_lib):
    # mattes.rs:1015 — the analytic derivative is the gradient of the value.
    p = small_pair(n=24, seed=5)
    g = _geo(oracle_lib, (24, 24, 24))
    c = [11.5, 11.5, 11.5]
    params = np.array([1.01, 0.02, 0.0, -0.01, 0.99, 0.01, 0.0, 0.0, 1.0, 0.3, -0.2, 0.1])
    r = oracle_lib.evaluate(p.fixed, g, p.moving, g, 32, 0, params, c)
    for k, h in [(9, 1e-4), (10, 1e-4), (0, 1e-6), (4, 1e-6)]:
        pp, pm = params.copy(), params.copy()
        pp[k] += h
        pm[k] -= h
        vp = oracle_lib.evaluate(p.fixed, g, p.moving, g, 32, 0, pp, c, derivative=False)["value"]
        vm = oracle_lib.evaluate(p.fixed, g, p.moving, g, 32, 0, pm, c, derivative=False)["value"]
        fd = (vp - vm) / (2 * h)
        scale = np.max(np.abs(r["derivative"]))
        assert abs(fd - r["derivative"][k]) <= 2e-3 * scale, (k, fd, r["derivative"][k])


def test_value_equals_evaluate_value(oracle_lib):
    # mattes.rs:1258, :1274 — the value-only walk and evaluate agree to the bit.
    p = small_pair()
    g = _geo(oracle_lib, (20, 20, 20))
    prm = [0.05, -0.02, 0.03, 0.5, -0.4, 0.2]
    a = oracle_lib.evaluate(p.fixed, g, p.moving, g, 50, 2, prm, [9.5, 9.5, 9.5], derivative=False)
    b = oracle_lib.evaluate(p.fixed, g, p.moving, g, 50, 2, prm, [9.5, 9.5, 9.5])
    assert a["value"] == b["value"] and a["valid"] == b["valid"]


def test_moving_mask_narrows_the_moving_axis(oracle_lib):
    # tests/mattes_mask.rs:95-134 — a masked-out bright voxel does not size the bins.
    p = small_pair()
    mov = p.moving.copy()
    mov[0, 0, 0] = 10000.0
    g = _geo(oracle_lib, (20, 20, 20))
    mask = np.ones_like(mov, dtype=np.uint8)
    mask[0, 0, 0] = 0
    a = oracle_lib.geometry_info(p.fixed, g, mov, g, 50)
    b = oracle_lib.geometry_info(p.fixed, g, mov, g, 50, mmask=mask)
    assert a["moving_max"] == 10000.0
    assert b["moving_max"] == float(p.moving.ravel()[1:].max()) or b["moving_max"] < 10000.0


def test_threaded_oracle_matches_serial(oracle_lib):
    p = small_pair(n=24, seed=9)
    g = _geo(oracle_lib, (24, 24, 24))
    prm = np.eye(3).ravel().tolist() + [0.2, 0.1, -0.3]
    a = oracle_lib.evaluate(p.fixed, g, p.moving, g, 50, 0, prm, [11.5] * 3)
    b = oracle_lib.evaluate(p.fixed, g, p.moving, g, 50, 0, prm, [11.5] * 3, nthreads=4)
    assert a["valid"] == b["valid"]
    assert abs(a["value"] - b["value"]) <= 1e-12 * abs(a["value"])
    assert np.allclose(a["derivative"], b["derivative"], rtol=1e-9, atol=1e-14)


# --- (3) two independent oracles agree ------------------------------------------

CASES = [
    # (name, n, kind, params, center, bins, sampling)
    ("affine_full", 20, 0, [1.02, 0.03, -0.01, -0.02, 0.98, 0.02, 0.01, -0.03, 1.01, 0.4, -0.3, 0.2], True, 50, None),
    ("versor_random", 24, 2, [0.03, -0.05, 0.02, 1.2, -0.7, 0.4], True, 32, ("random", 0.3, 11)),
    ("euler_regular", 20, 1, [0.04, 0.02, -0.06, -0.5, 0.8, 0.1], True, 64, ("regular", 0.2, 0)),
    ("translation_identity", 20, 3, [0.0, 0.0, 0.0], False, 50, None),
]


@pytest.mark.parametrize("name,n,kind,params,centered,bins,sampling", CASES)
def test_numpy_oracle_agrees(oracle_lib, name, n, kind, params, centered, bins, sampling):
    p = small_pair(n=n, seed=13)
    spacing = (1.0, 1.1, 0.9)
    origin = (-2.0, 1.5, 0.25)
    g = _geo(oracle_lib, (n, n, n), spacing=spacing, origin=origin)
    gd = geo_dict((n, n, n), spacing=spacing, origin=origin)
    center = [origin[d] + spacing[d] * (n - 1) / 2 for d in range(3)] if centered else None
    draw = None
    if sampling:
        strat = {"regular": 1, "random": 2}[sampling[0]]
        draw = oracle_lib.draw_samples(n ** 3, strat, sampling[1], sampling[2])
    mmask = (p.moving > np.percentile(p.moving, 5)).astype(np.uint8) if name == "versor_random" else None
    a = oracle_lib.evaluate(p.fixed, g, p.moving, g, bins, kind, params, center, draw=draw,
                            mmask=mmask, per_sample=True, histogram=True)
    b = np_oracle.evaluate(p.fixed, gd, p.moving, gd, bins, kind, params, center, draw=draw, mmask=mmask)
    np.testing.assert_array_equal(a["status"], b["status"])
    np.testing.assert_array_equal(a["fi"], b["fi"])
    np.testing.assert_array_equal(a["mi"], b["mi"])
    assert a["valid"] == b["valid"] > 0
    np.testing.assert_array_equal(a["joint"], b["joint"])
    assert a["value"] == b["value"]
    scale = np.max(np.abs(a["derivative"]))
    assert np.max(np.abs(a["derivative"] - b["derivative"])) <= 1e-12 * scale
