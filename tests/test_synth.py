"""The counter-based synthetic pair: seeded and reproducible on the CPU, and the
device generator (mi_synth_pair) equal to it within the rounding of exp/log/cos.
"""
import numpy as np
import pytest


def test_counter_noise_is_reproducible_and_standard_normal():
    from sitk_b200 import synth
    k = synth.noise_key(20261203, 1)
    a = synth.counter_normal(k, 400_000)
    np.testing.assert_array_equal(a, synth.counter_normal(k, 400_000))
    assert abs(a.mean()) < 0.01 and abs(a.std() - 1.0) < 0.01
    # the two fields of a pair are different streams
    b = synth.counter_normal(synth.noise_key(20261203, 2), 1000)
    assert not np.allclose(a[:1000], b)


def test_counter_pair_is_reproducible_from_its_seed():
    from sitk_b200 import synth
    p = synth.make_pair_counter(24, 5, 123, 8.0, 3.0)
    q = synth.make_pair_counter(24, 5, 123, 8.0, 3.0)
    np.testing.assert_array_equal(p.fixed, q.fixed)
    np.testing.assert_array_equal(p.moving, q.moving)
    r = synth.make_pair_counter(24, 5, 124, 8.0, 3.0)
    assert not np.array_equal(p.fixed, r.fixed)


@pytest.mark.gpu
@pytest.mark.parametrize("n,seed", [(24, 5), (37, 99), (64, 20261203)])
def test_device_generator_equals_the_cpu_generator(n, seed):
    from sitk_b200 import synth
    cpu = synth.make_pair_counter(n, 12, seed, 10.0, 5.0)
    f, m, truth = synth.make_pair_device(n, 12, seed, 10.0, 5.0)
    np.testing.assert_array_equal(truth.matrix, cpu.matrix)
    df, dm = f.to_host(), m.to_host()
    # FP64 throughout on both sides; exp/log/cos may differ in the last bit, which can
    # move the f32 result by one unit at most
    for d, c in ((df, cpu.fixed), (dm, cpu.moving)):
        ulp = np.spacing(np.abs(c).astype(np.float32))
        assert np.all(np.abs(d - c) <= ulp)
        assert np.mean(d == c) > 0.99
