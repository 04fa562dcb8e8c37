"""CPU tests of the C ABI: the library loads, exports every declared symbol, and its
host-side transform code forms the reference's stage bit for bit (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def _declared():
    src = open(os.path.join(ROOT, "include", "mi_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mi_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from sitk_b200 import _lib
    L = _lib.load()
    declared = _declared()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(L, name), name
    assert set(declared) <= set(_lib.EXPORTED)


def test_status_strings_name_every_refusal():
    from sitk_b200 import _lib
    L = _lib.load()
    for code, name in _lib.STATUS_NAMES.items():
        s = L.mi_status_string(code).decode()
        assert s and s != "unknown status", name


def test_no_device_is_reported_by_name():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from sitk_b200 import _lib
    L = _lib.load()
    h = ctypes.c_void_p()
    assert L.mi_context_create(0, ctypes.byref(h)) == 2  # MI_ERR_NO_DEVICE


FAMILIES = [
    (0, [1.02, 0.03, -0.01, -0.02, 0.98, 0.02, 0.01, -0.03, 1.01, 0.4, -0.3, 0.2], [10.5, -3.25, 7.0]),
    (1, [0.04, 0.02, -0.06, -0.5, 0.8, 0.1], [10.5, -3.25, 7.0]),
    (1, [0.04, 0.02, -0.06, -0.5, 0.8, 0.1], [10.5, -3.25, 7.0, 1.0]),
    (2, [0.03, -0.05, 0.02, 1.2, -0.7, 0.4], [127.5, 127.5, 127.5]),
    (2, [0.7, 0.6, 0.5, 1.2, -0.7, 0.4], [1.0, 2.0, 3.0]),  # norm ≥ 1: rescaled below 1
    (3, [0.3, -0.2, 0.1], []),
]


@pytest.mark.parametrize("kind,params,fixed", FAMILIES)
def test_transform_stage_is_the_oracles_to_the_bit(oracle_lib, kind, params, fixed):
    from sitk_b200 import metric, transforms
    cls = {0: transforms.AffineTransform, 1: transforms.Euler3DTransform,
           2: transforms.VersorRigid3DTransform, 3: transforms.TranslationTransform}[kind]
    t = cls.__new__(cls)
    transforms.ParametricTransform.__init__(t, params, fixed)
    st, j0, jc = metric.transform_form(t)
    ref = oracle_lib.transform(kind, params, fixed if fixed else None, point=[3.0, -4.0, 5.5])
    np.testing.assert_array_equal(st[:9], ref["matrix"].ravel())
    np.testing.assert_array_equal(st[9:], ref["offset"])
    # the Jacobian's affine form reproduces the oracle's per-point Jacobian
    x = np.array([3.0, -4.0, 5.5])
    jx = j0 + sum(x[e] * jc[e] for e in range(3))
    np.testing.assert_allclose(jx, ref["jacobian"], rtol=1e-12, atol=1e-12)


def test_fastdiv_multiplier_divides_exactly():
    # csrc/internal.h make_fastdiv + sampler.cuh fdiv: q = (umulhi(n, m) + n) >> s
    rng = np.random.default_rng(0)
    divisors = [1, 2, 3, 5, 7, 48, 64, 100, 127, 192, 255, 256, 257, 511, 512, 1000, 4093, 65535, 65536]
    ns = np.concatenate([rng.integers(0, 2 ** 32, 20000, dtype=np.uint64),
                         np.array([0, 1, 2 ** 32 - 1, 2 ** 31, 2 ** 24 - 1, 2 ** 24], dtype=np.uint64)])
    for d in divisors:
        s = 0
        while (1 << s) < d:
            s += 1
        m = ((1 << 32) * ((1 << s) - d)) // d + 1
        assert m < (1 << 32)
        for n in ns.tolist():
            q = (((n * m) >> 32) + n) >> s
            assert q == n // d, (n, d)
