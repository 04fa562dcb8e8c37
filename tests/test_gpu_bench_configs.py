"""Parity at the configurations the benchmark and the workload list name (needs a B200).

Each case is held to the same contract as tests/test_gpu_parity.py (the reference's
device pins, tests/mattes_device.rs:189-350): every sample's validity and both Parzen
bins equal the oracle's exactly, the value within 1e-5 relative, every derivative
component within 1e-4 of max|∂|.

- the benchmark's own workload: the 256³ VersorRigid3D pair, 32 bins, 10 % SplitMix64
  samples, at the benchmark's pose (bench.py's constants, imported, not restated);
- the 512³ Euler3D case with 64 bins and 20 % samples, with the moving volume stored as
  f32 (against the oracle on the f32 volume) and as BF16 (against the oracle on the
  rounded volume, the values the device samples);
- the 64³ affine case (50 bins, the whole grid) over a 100-iteration regular-step
  gradient descent with physical-shift scales: every evaluation the device driver
  makes is checked against the oracle at the same parameters, and every step against
  the update rule applied to the device's own derivative;
- a six-stage point map (the reference replays up to eight, cuda/ops/resident.rs:74)
  against the oracle's stage-by-stage replay, and the refusal of 0 and 9 stages.
"""
import importlib.util
import os

import numpy as np
import pytest

from conftest import ROOT, small_pair
from test_gpu_parity import VALUE_RTOL, DERIV_RTOL, _compare
from test_registration import _corner_jacobians, _replay_rsgd, _shift_scales_and_lr

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def _bench():
    spec = importlib.util.spec_from_file_location("bench_constants", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_bench_workload_256cubed_versor_random10(oracle_lib):
    import sitk_b200 as sb
    B = _bench()
    pair = B.make_workload(B.SEED)
    t = sb.VersorRigid3DTransform(B.POSE[:3], B.POSE[3:], [(B.N - 1) / 2.0] * 3)
    metric, mv, ref, dec = _compare(oracle_lib, pair, B.N, t, B.BINS, strategy=2, pct=B.PCT, seed=B.SEED,
                                    nthreads=THREADS)
    assert metric.info()["n_samples"] == int(B.N ** 3 * B.PCT)
    assert mv.valid_points > 0.9 * metric.info()["n_samples"]
    # the fast path decides nearly every sample of this generic pose
    assert dec["exact"].mean() < 0.05


@pytest.mark.parametrize("storage", ["f32", "bf16"])
def test_config3_512cubed_euler_64_bins(oracle_lib, storage):
    import sitk_b200 as sb
    from sitk_b200 import synth
    n = 512
    ctx = sb.Context(0)
    f, m, _ = synth.make_pair_device(n, 120, 20261203 + 3, 10.0, 5.0, None, ctx=ctx)
    p = synth.Pair(f.to_host(), m.to_host(), np.eye(3), np.zeros(3), np.zeros(3))
    f.free()
    m.free()
    c = [(n - 1) / 2.0] * 3
    t = sb.Euler3DTransform((0.02, -0.015, 0.03), (0.8, -0.6, 0.4), c)
    metric, mv, ref, _ = _compare(oracle_lib, p, n, t, 64, strategy=2, pct=0.2, seed=20261203,
                                  moving_storage=storage, nthreads=THREADS, other_form=False)
    assert metric.info()["n_samples"] == int(n ** 3 * 0.2)
    if storage == "bf16":
        # the storage error itself, against the oracle on the f32 volume: reported by
        # the storage study, bounded loosely here
        g = oracle_lib.make_geometry((n, n, n))
        draw = oracle_lib.draw_samples(n ** 3, 2, 0.2, 20261203)
        ref_f = oracle_lib.evaluate(p.fixed, g, p.moving, g, 64, t.kind, t.params, t.fixed_params, draw=draw,
                                    nthreads=THREADS)
        assert abs(mv.value - ref_f["value"]) <= 1e-3 * abs(ref_f["value"])
        assert np.max(np.abs(mv.derivative - ref_f["derivative"])) <= 0.05 * np.max(np.abs(ref_f["derivative"]))


def test_config0_affine_100_iterations_every_step_checked(oracle_lib):
    import sitk_b200 as sb
    from sitk_b200 import registration, synth
    n = 64
    p = synth.config0_pair()
    geo = oracle_lib.make_geometry((n, n, n))
    f = sb.DeviceImage.upload(p.fixed)
    m = sb.DeviceImage.upload(p.moving)
    metric = sb.DeviceMattesMetric.from_device(f, m, 50)
    fp = np.array([(n - 1) / 2.0] * 3)
    t = sb.AffineTransform(np.eye(3), (0.0, 0.0, 0.0), fp)
    start = t.params.copy()
    res = registration.register_rsgd(metric, t, iterations=100, record=True)
    tr = res.trace
    P = 12
    assert len(tr) == res.evaluations and res.evaluations >= 30
    for row in tr:
        o = oracle_lib.evaluate(p.fixed, geo, p.moving, geo, 50, 0, row[1:1 + P], fp, nthreads=THREADS)
        assert abs(row[0] - o["value"]) <= VALUE_RTOL * abs(o["value"])
        d = o["derivative"]
        assert np.max(np.abs(row[1 + P:] - d)) <= DERIV_RTOL * np.max(np.abs(d))
    jac, min_sp = _corner_jacobians(oracle_lib, 0, start, fp, geo)
    scales, lr = _shift_scales_and_lr(jac, min_sp, tr[0, 1 + P:])
    pred = _replay_rsgd(tr, P, scales, lr)
    np.testing.assert_allclose(tr[1:, 1:1 + P], pred, rtol=0, atol=1e-9)
    # the oracle's own 100-iteration run lands in the same place
    ref = oracle_lib.register(p.fixed, geo, p.moving, geo, 50, 0, start, fp, iterations=100, nthreads=THREADS)
    assert abs(res.value - ref["value"]) <= 2e-3 * abs(ref["value"])
    assert res.trace[-1, 0] < res.trace[0, 0]


def _compose_stage(a, b):
    """The stage a ∘ b as one 12-double stage (for building the Jacobian form only)."""
    Ma, ta = a[:9].reshape(3, 3), a[9:]
    Mb, tb = b[:9].reshape(3, 3), b[9:]
    return np.concatenate([(Ma @ Mb).ravel(), Ma @ tb + ta])


def test_six_stage_point_map_and_stage_count_refusals(oracle_lib):
    import sitk_b200 as sb
    from sitk_b200.metric import transform_form
    n = 40
    p = small_pair(n=n, seed=61, rot=6.0, trans=3.0)
    f = sb.DeviceImage.upload(p.fixed)
    m = sb.DeviceImage.upload(p.moving)
    metric = sb.DeviceMattesMetric.from_device_sampled(f, m, bins=32, strategy=sb.SAMPLING_RANDOM, percentage=0.5,
                                                       seed=5)
    c = [(n - 1) / 2.0] * 3
    opt = sb.AffineTransform(np.eye(3) + 0.01 * np.array([[1, -2, 0], [1, 1, 0], [0, 2, -1]]), (0.3, -0.4, 0.2), c)
    s0, j0, jc = transform_form(opt)
    rng = np.random.default_rng(8)
    stages = [s0]
    for _ in range(5):
        ang = rng.uniform(-0.02, 0.02, 3)
        cz, sz = np.cos(ang[2]), np.sin(ang[2])
        R = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]]) @ np.diag(1 + rng.uniform(-0.01, 0.01, 3))
        stages.append(np.concatenate([R.ravel(), rng.uniform(-0.5, 0.5, 3)]))
    # J of the composite w.r.t. the first stage's parameters: the later stages' matrices
    # times the first stage's Jacobian form (still affine in the point)
    chain = np.eye(3)
    for s in stages[1:]:
        chain = s[:9].reshape(3, 3) @ chain
    J0 = chain @ j0
    JC = np.stack([chain @ jc[e] for e in range(3)])
    st = np.concatenate(stages)
    mv = metric.evaluate_stages(st, J0, JC)
    geo = oracle_lib.make_geometry((n, n, n))
    draw = oracle_lib.draw_samples(n ** 3, 2, 0.5, 5)
    ref = oracle_lib.evaluate_stages(p.fixed, geo, p.moving, geo, 32, st, J0, JC, draw=draw, per_sample=True)
    assert mv.valid_points == ref["valid"]
    assert abs(mv.value - ref["value"]) <= VALUE_RTOL * abs(ref["value"])
    assert np.max(np.abs(mv.derivative - ref["derivative"])) <= DERIV_RTOL * np.max(np.abs(ref["derivative"]))
    # per-sample decisions, matched voxel for voxel
    dec = metric.sample_decisions(st)
    dev = np.asarray(dec["flat"], dtype=np.int64)
    o_ord = np.argsort(draw, kind="stable")
    d_ord = np.argsort(dev, kind="stable")
    order = np.empty_like(o_ord)
    order[d_ord] = o_ord
    np.testing.assert_array_equal(dec["status"], ref["status"][order])
    np.testing.assert_array_equal(dec["mi"], np.where(ref["status"][order] == 2, ref["mi"][order], -1))
    # the same map folded into one stage gives the same valid count (the decisions of a
    # folded map may differ in the last bits, so only the count's size is compared)
    one = stages[0]
    for s in stages[1:]:
        one = _compose_stage(s, one)
    v1, n1 = metric.value_stages(one)
    assert abs(n1 - mv.valid_points) <= 0.001 * mv.valid_points
    # an empty map and one of nine stages are refused by name (resident.rs:698-703)
    for bad in (np.zeros(0), np.zeros(12 * 9)):
        with pytest.raises(sb.MiError) as e:
            metric.value_stages(bad)
        assert e.value.name == "MI_ERR_POINT_MAP_STAGE_COUNT"
        with pytest.raises(sb.MiError) as e:
            metric.evaluate_stages(bad, J0, JC)
        assert e.value.name == "MI_ERR_POINT_MAP_STAGE_COUNT"
    # eight stages are accepted
    v8, n8 = metric.value_stages(np.concatenate(stages + stages[1:3]))
    assert n8 > 0 and np.isfinite(v8)
