"""ctypes front end of the CPU oracle (test infrastructure only).

The oracle restates the reference's CPU Mattes metric (crates/sitk/src/registration/
mattes.rs:442-676 and the helpers it calls) in serial FP64 C++; see
oracle/mattes_oracle.cpp for the per-function citations and the parity status
("parity unpinned": the Rust reference cannot be built here). Only tests/, the
smoke check and bench.py's CPU-baseline legs import this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmattes_oracle.so")

AFFINE, EULER3D, VERSOR_RIGID3D, TRANSLATION = 0, 1, 2, 3
NPARAMS = {AFFINE: 12, EULER3D: 6, VERSOR_RIGID3D: 6, TRANSLATION: 3}

STATUS = {0: "ok", 1: "too few bins", 2: "constant fixed", 3: "constant moving",
          4: "singular direction", 5: "bad argument"}


class OrGeometry(ctypes.Structure):
    _fields_ = [("size", ctypes.c_int64 * 3), ("spacing", ctypes.c_double * 3),
                ("origin", ctypes.c_double * 3), ("direction", ctypes.c_double * 9)]


def make_geometry(size, spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0),
                  direction=(1, 0, 0, 0, 1, 0, 0, 0, 1)) -> OrGeometry:
    g = OrGeometry()
    for i in range(3):
        g.size[i] = int(size[i])
        g.spacing[i] = float(spacing[i])
        g.origin[i] = float(origin[i])
    for i in range(9):
        g.direction[i] = float(direction[i])
    return g


def build() -> str:
    """Compile the oracle library with its Makefile (g++, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    L = ctypes.CDLL(LIB_PATH)
    P = ctypes.POINTER
    dp, fp, i64p = P(ctypes.c_double), P(ctypes.c_float), P(ctypes.c_int64)
    u8p, i8p, i32p = P(ctypes.c_uint8), P(ctypes.c_int8), P(ctypes.c_int32)
    gp = P(OrGeometry)
    L.or_splitmix64_next.argtypes = [P(ctypes.c_uint64)]
    L.or_splitmix64_next.restype = ctypes.c_uint64
    L.or_draw_samples.argtypes = [ctypes.c_int64, ctypes.c_int, ctypes.c_double, ctypes.c_uint64,
                                  i64p, ctypes.c_int64]
    L.or_draw_samples.restype = ctypes.c_int64
    L.or_metric_geometry.argtypes = [fp, gp, fp, gp, u8p, u8p, i64p, ctypes.c_int64, ctypes.c_int,
                                     dp, i64p]
    L.or_metric_geometry.restype = ctypes.c_int
    L.or_mattes_evaluate.argtypes = [fp, gp, fp, gp, u8p, u8p, i64p, ctypes.c_int64, ctypes.c_int,
                                     ctypes.c_int, dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     dp, dp, i64p, i8p, i32p, i32p, dp, dp]
    L.or_mattes_evaluate.restype = ctypes.c_int
    L.or_mattes_evaluate_stages.argtypes = [fp, gp, fp, gp, u8p, u8p, i64p, ctypes.c_int64, ctypes.c_int, dp,
                                            ctypes.c_int, dp, dp, ctypes.c_int, ctypes.c_int, dp, dp, i64p, i8p,
                                            i32p, i32p]
    L.or_mattes_evaluate_stages.restype = ctypes.c_int
    L.or_transform.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int, dp, dp, dp, dp, dp]
    L.or_transform.restype = ctypes.c_int
    L.or_cubic_bspline.argtypes = [dp, dp, dp, ctypes.c_int64]
    L.or_cubic_bspline.restype = ctypes.c_int
    L.or_kahan_sum.argtypes = [dp, ctypes.c_int64]
    L.or_kahan_sum.restype = ctypes.c_double
    L.or_round_half_integer_up.argtypes = [ctypes.c_double]
    L.or_round_half_integer_up.restype = ctypes.c_int64
    L.or_invert3.argtypes = [dp, dp]
    L.or_invert3.restype = ctypes.c_int
    for name in ("or_ms_evaluate", "or_ncc_evaluate"):
        f = getattr(L, name)
        f.argtypes = [fp, gp, fp, gp, u8p, u8p, i64p, ctypes.c_int64, ctypes.c_int, dp, dp, ctypes.c_int,
                      ctypes.c_int, dp, dp, i64p]
        f.restype = ctypes.c_int
    _lib = L
    return L


def _ptr(a, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctype))


class OracleError(RuntimeError):
    def __init__(self, code):
        super().__init__(f"oracle refused: {STATUS.get(code, code)}")
        self.code = code


def splitmix64(seed: int, n: int) -> list[int]:
    st = ctypes.c_uint64(seed)
    return [lib().or_splitmix64_next(ctypes.byref(st)) for _ in range(n)]


def draw_samples(voxels: int, strategy: int, percentage: float, seed: int):
    """metric.rs:419-437 — None (strategy 0) returns None; 1 Regular; 2 Random."""
    n = lib().or_draw_samples(voxels, strategy, percentage, seed, None, 0)
    if n < 0:
        return None
    out = np.empty(n, dtype=np.int64)
    lib().or_draw_samples(voxels, strategy, percentage, seed, _ptr(out, ctypes.c_int64), n)
    return out


def geometry_info(fixed, fgeo, moving, mgeo, bins, fmask=None, mmask=None, draw=None):
    fixed = np.ascontiguousarray(fixed, dtype=np.float32)
    moving = np.ascontiguousarray(moving, dtype=np.float32)
    fm = None if fmask is None else np.ascontiguousarray(fmask, dtype=np.uint8)
    mm = None if mmask is None else np.ascontiguousarray(mmask, dtype=np.uint8)
    dr = None if draw is None else np.ascontiguousarray(draw, dtype=np.int64)
    out = np.zeros(8)
    ns = ctypes.c_int64(0)
    st = lib().or_metric_geometry(_ptr(fixed, ctypes.c_float), ctypes.byref(fgeo),
                                  _ptr(moving, ctypes.c_float), ctypes.byref(mgeo),
                                  _ptr(fm, ctypes.c_uint8), _ptr(mm, ctypes.c_uint8),
                                  _ptr(dr, ctypes.c_int64), 0 if dr is None else len(dr), bins,
                                  _ptr(out, ctypes.c_double), ctypes.byref(ns))
    if st:
        raise OracleError(st)
    keys = ["fixed_min", "fixed_max", "moving_min", "moving_max", "fixed_bin_size",
            "moving_bin_size", "fixed_normalized_min", "moving_normalized_min"]
    d = dict(zip(keys, out.tolist()))
    d["nsamples"] = ns.value
    return d


def evaluate(fixed, fgeo, moving, mgeo, bins, kind, params, fixed_params=None, fmask=None,
             mmask=None, draw=None, derivative=True, nthreads=1, per_sample=False,
             histogram=False):
    """value = −MI and derivative (mattes.rs:522-676); returns a dict."""
    fixed = np.ascontiguousarray(fixed, dtype=np.float32)
    moving = np.ascontiguousarray(moving, dtype=np.float32)
    fm = None if fmask is None else np.ascontiguousarray(fmask, dtype=np.uint8)
    mm = None if mmask is None else np.ascontiguousarray(mmask, dtype=np.uint8)
    dr = None if draw is None else np.ascontiguousarray(draw, dtype=np.int64)
    params = np.ascontiguousarray(params, dtype=np.float64)
    fpar = None if fixed_params is None else np.ascontiguousarray(fixed_params, dtype=np.float64)
    nparams = NPARAMS[kind]
    deriv = np.zeros(nparams)
    value = ctypes.c_double(0.0)
    valid = ctypes.c_int64(0)
    status = fi = mi = None
    if per_sample:
        nvox = int(np.prod([fgeo.size[i] for i in range(3)]))
        n = nvox if dr is None else len(dr)
        status = np.full(n, -1, dtype=np.int8)
        fi = np.full(n, -1, dtype=np.int32)
        mi = np.full(n, -1, dtype=np.int32)
    joint = margin = None
    if histogram:
        joint = np.zeros(bins * bins)
        margin = np.zeros(bins)
    st = lib().or_mattes_evaluate(
        _ptr(fixed, ctypes.c_float), ctypes.byref(fgeo), _ptr(moving, ctypes.c_float),
        ctypes.byref(mgeo), _ptr(fm, ctypes.c_uint8), _ptr(mm, ctypes.c_uint8),
        _ptr(dr, ctypes.c_int64), 0 if dr is None else len(dr), bins, kind,
        _ptr(params, ctypes.c_double), _ptr(fpar, ctypes.c_double),
        0 if fpar is None else len(fpar), 1 if derivative else 0, nthreads,
        ctypes.byref(value), _ptr(deriv, ctypes.c_double), ctypes.byref(valid),
        _ptr(status, ctypes.c_int8), _ptr(fi, ctypes.c_int32), _ptr(mi, ctypes.c_int32),
        _ptr(joint, ctypes.c_double), _ptr(margin, ctypes.c_double))
    if st:
        raise OracleError(st)
    out = {"value": value.value, "derivative": deriv, "valid": valid.value}
    if per_sample:
        out.update(status=status, fi=fi, mi=mi)
    if histogram:
        out.update(joint=joint, fixed_marginal=margin)
    return out


def evaluate_stages(fixed, fgeo, moving, mgeo, bins, stages, jac0, jacc, fmask=None, mmask=None, draw=None,
                    nthreads=1, per_sample=False):
    """value and derivative at a point map of 1..8 stages (12 doubles each, replayed in
    order, matrix_offset.rs:102-109) with the Jacobian J(x) = jac0 + Σ_e x_e·jacc[e]
    (jac0 3×P row-major, jacc three such blocks)."""
    fixed = np.ascontiguousarray(fixed, dtype=np.float32)
    moving = np.ascontiguousarray(moving, dtype=np.float32)
    fm = None if fmask is None else np.ascontiguousarray(fmask, dtype=np.uint8)
    mm = None if mmask is None else np.ascontiguousarray(mmask, dtype=np.uint8)
    dr = None if draw is None else np.ascontiguousarray(draw, dtype=np.int64)
    st = np.ascontiguousarray(stages, dtype=np.float64).ravel()
    j0 = np.ascontiguousarray(jac0, dtype=np.float64).ravel()
    jc = np.ascontiguousarray(jacc, dtype=np.float64).ravel()
    nparams = j0.size // 3
    deriv = np.zeros(nparams)
    value = ctypes.c_double(0.0)
    valid = ctypes.c_int64(0)
    status = fi = mi = None
    if per_sample:
        nvox = int(np.prod([fgeo.size[i] for i in range(3)]))
        n = nvox if dr is None else len(dr)
        status = np.full(n, -1, dtype=np.int8)
        fi = np.full(n, -1, dtype=np.int32)
        mi = np.full(n, -1, dtype=np.int32)
    r = lib().or_mattes_evaluate_stages(
        _ptr(fixed, ctypes.c_float), ctypes.byref(fgeo), _ptr(moving, ctypes.c_float), ctypes.byref(mgeo),
        _ptr(fm, ctypes.c_uint8), _ptr(mm, ctypes.c_uint8), _ptr(dr, ctypes.c_int64), 0 if dr is None else len(dr),
        bins, _ptr(st, ctypes.c_double), st.size // 12, _ptr(j0, ctypes.c_double), _ptr(jc, ctypes.c_double),
        nparams, nthreads, ctypes.byref(value), _ptr(deriv, ctypes.c_double), ctypes.byref(valid),
        _ptr(status, ctypes.c_int8), _ptr(fi, ctypes.c_int32), _ptr(mi, ctypes.c_int32))
    if r:
        raise OracleError(r)
    out = {"value": value.value, "derivative": deriv, "valid": valid.value}
    if per_sample:
        out.update(status=status, fi=fi, mi=mi)
    return out


def _moments_metric(fn, fixed, fgeo, moving, mgeo, kind, params, fixed_params, fmask, mmask, draw, derivative):
    fixed = np.ascontiguousarray(fixed, dtype=np.float32)
    moving = np.ascontiguousarray(moving, dtype=np.float32)
    fm = None if fmask is None else np.ascontiguousarray(np.asarray(fmask) != 0, dtype=np.uint8)
    mm = None if mmask is None else np.ascontiguousarray(np.asarray(mmask) != 0, dtype=np.uint8)
    dr = None if draw is None else np.ascontiguousarray(draw, dtype=np.int64)
    params = np.ascontiguousarray(params, dtype=np.float64)
    fpar = None if fixed_params is None else np.ascontiguousarray(fixed_params, dtype=np.float64)
    deriv = np.zeros(NPARAMS[kind])
    value = ctypes.c_double(0.0)
    valid = ctypes.c_int64(0)
    st = fn(_ptr(fixed, ctypes.c_float), ctypes.byref(fgeo), _ptr(moving, ctypes.c_float), ctypes.byref(mgeo),
            _ptr(fm, ctypes.c_uint8), _ptr(mm, ctypes.c_uint8), _ptr(dr, ctypes.c_int64),
            0 if dr is None else len(dr), kind, _ptr(params, ctypes.c_double), _ptr(fpar, ctypes.c_double),
            0 if fpar is None else len(fpar), 1 if derivative else 0, ctypes.byref(value),
            _ptr(deriv, ctypes.c_double), ctypes.byref(valid))
    if st:
        raise OracleError(st)
    return {"value": value.value, "derivative": deriv, "valid": valid.value}


def mean_squares(fixed, fgeo, moving, mgeo, kind, params, fixed_params=None, fmask=None, mmask=None, draw=None,
                 derivative=True):
    """CpuBackend::mean_squares / mean_squares_value (registration/metric.rs:1064-1196)."""
    return _moments_metric(lib().or_ms_evaluate, fixed, fgeo, moving, mgeo, kind, params, fixed_params, fmask,
                           mmask, draw, derivative)


def correlation(fixed, fgeo, moving, mgeo, kind, params, fixed_params=None, fmask=None, mmask=None, draw=None,
                derivative=True):
    """CorrelationMetric::evaluate / value (registration/correlation.rs:200-410)."""
    return _moments_metric(lib().or_ncc_evaluate, fixed, fgeo, moving, mgeo, kind, params, fixed_params, fmask,
                           mmask, draw, derivative)


def _bs_bind():
    L = lib()
    if not hasattr(L.or_bspline_mattes_evaluate, "_typed"):
        P = ctypes.POINTER
        dp, fp, i64p = P(ctypes.c_double), P(ctypes.c_float), P(ctypes.c_int64)
        L.or_bspline_transform_point.argtypes = [dp, dp, ctypes.c_int64, dp, dp]
        L.or_bspline_transform_point.restype = ctypes.c_int
        L.or_bspline_mattes_evaluate.argtypes = [fp, P(OrGeometry), fp, P(OrGeometry), P(ctypes.c_uint8),
                                                 P(ctypes.c_uint8), i64p, ctypes.c_int64, ctypes.c_int, dp, dp,
                                                 ctypes.c_int64, ctypes.c_int, dp, dp, i64p, P(ctypes.c_int8),
                                                 P(ctypes.c_int32), P(ctypes.c_int32)]
        L.or_bspline_mattes_evaluate.restype = ctypes.c_int
        L.or_bspline_mattes_evaluate._typed = True
    return L


def bspline_transform_point(fixed18, coef, point):
    """BSplineTransform::transform_point (transform/bspline.rs:561-585)."""
    f = np.ascontiguousarray(fixed18, dtype=np.float64)
    c = np.ascontiguousarray(coef, dtype=np.float64)
    x = np.ascontiguousarray(point, dtype=np.float64)
    y = np.zeros(3)
    st = _bs_bind().or_bspline_transform_point(_ptr(f, ctypes.c_double), _ptr(c, ctypes.c_double), c.size,
                                               _ptr(x, ctypes.c_double), _ptr(y, ctypes.c_double))
    if st:
        raise OracleError(st)
    return y


def bspline_mattes(fixed, fgeo, moving, mgeo, bins, fixed18, coef, fmask=None, mmask=None, draw=None,
                   derivative=True, per_sample=False):
    """Mattes value and derivative through a B-spline transform: evaluate_sparse_support
    (registration/mattes.rs:722-796)."""
    fixed = np.ascontiguousarray(fixed, dtype=np.float32)
    moving = np.ascontiguousarray(moving, dtype=np.float32)
    fm = None if fmask is None else np.ascontiguousarray(np.asarray(fmask) != 0, dtype=np.uint8)
    mm = None if mmask is None else np.ascontiguousarray(np.asarray(mmask) != 0, dtype=np.uint8)
    dr = None if draw is None else np.ascontiguousarray(draw, dtype=np.int64)
    f18 = np.ascontiguousarray(fixed18, dtype=np.float64)
    c = np.ascontiguousarray(coef, dtype=np.float64)
    deriv = np.zeros(c.size)
    value = ctypes.c_double(0.0)
    valid = ctypes.c_int64(0)
    status = fi = mi = None
    if per_sample:
        nvox = int(np.prod([fgeo.size[i] for i in range(3)]))
        n = nvox if dr is None else len(dr)
        status = np.full(n, -1, dtype=np.int8)
        fi = np.full(n, -1, dtype=np.int32)
        mi = np.full(n, -1, dtype=np.int32)
    st = _bs_bind().or_bspline_mattes_evaluate(
        _ptr(fixed, ctypes.c_float), ctypes.byref(fgeo), _ptr(moving, ctypes.c_float), ctypes.byref(mgeo),
        _ptr(fm, ctypes.c_uint8), _ptr(mm, ctypes.c_uint8), _ptr(dr, ctypes.c_int64), 0 if dr is None else len(dr),
        bins, _ptr(f18, ctypes.c_double), _ptr(c, ctypes.c_double), c.size, 1 if derivative else 0,
        ctypes.byref(value), _ptr(deriv, ctypes.c_double), ctypes.byref(valid), _ptr(status, ctypes.c_int8),
        _ptr(fi, ctypes.c_int32), _ptr(mi, ctypes.c_int32))
    if st:
        raise OracleError(st)
    out = {"value": value.value, "derivative": deriv, "valid": valid.value}
    if per_sample:
        out.update(status=status, fi=fi, mi=mi)
    return out


def transform(kind, params, fixed_params=None, point=None):
    params = np.ascontiguousarray(params, dtype=np.float64)
    fpar = None if fixed_params is None else np.ascontiguousarray(fixed_params, dtype=np.float64)
    m = np.zeros(9)
    o = np.zeros(3)
    jac = np.zeros(3 * NPARAMS[kind])
    mapped = np.zeros(3)
    pt = None if point is None else np.ascontiguousarray(point, dtype=np.float64)
    st = lib().or_transform(kind, _ptr(params, ctypes.c_double), _ptr(fpar, ctypes.c_double),
                            0 if fpar is None else len(fpar), _ptr(pt, ctypes.c_double),
                            _ptr(m, ctypes.c_double), _ptr(o, ctypes.c_double),
                            _ptr(jac, ctypes.c_double), _ptr(mapped, ctypes.c_double))
    if st:
        raise OracleError(st)
    return {"matrix": m.reshape(3, 3), "offset": o,
            "jacobian": jac.reshape(3, NPARAMS[kind]), "mapped": mapped}


def cubic_bspline(u):
    u = np.ascontiguousarray(u, dtype=np.float64)
    v = np.zeros_like(u)
    d = np.zeros_like(u)
    lib().or_cubic_bspline(_ptr(u, ctypes.c_double), _ptr(v, ctypes.c_double),
                           _ptr(d, ctypes.c_double), u.size)
    return v, d


def kahan_sum(v):
    v = np.ascontiguousarray(v, dtype=np.float64)
    return lib().or_kahan_sum(_ptr(v, ctypes.c_double), v.size)


def round_half_integer_up(x: float) -> int:
    return lib().or_round_half_integer_up(x)


def register(fixed, fgeo, moving, mgeo, bins, kind, params, fixed_params=None, fmask=None,
             mmask=None, draw=None, iterations=100, minimum_step=1e-4, gradient_tolerance=1e-4,
             relaxation=0.5, learning_rate=1.0, estimate_learning_rate=True, shift_scales=True,
             nthreads=1):
    """One level of regular-step gradient descent with physical-shift scales
    (registration/optimizer.rs:352-440, scales.rs:572-871, method.rs:3140-3400)."""
    L = lib()
    if not hasattr(L.or_register, "_typed"):
        P = ctypes.POINTER
        dp = P(ctypes.c_double)
        L.or_register.argtypes = [P(ctypes.c_float), P(OrGeometry), P(ctypes.c_float), P(OrGeometry),
                                  P(ctypes.c_uint8), P(ctypes.c_uint8), P(ctypes.c_int64), ctypes.c_int64,
                                  ctypes.c_int, ctypes.c_int, dp, dp, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, P(ctypes.c_int),
                                  P(ctypes.c_int)]
        L.or_register.restype = ctypes.c_int
        L.or_register._typed = True
    fixed = np.ascontiguousarray(fixed, dtype=np.float32)
    moving = np.ascontiguousarray(moving, dtype=np.float32)
    fm = None if fmask is None else np.ascontiguousarray(fmask, dtype=np.uint8)
    mm = None if mmask is None else np.ascontiguousarray(mmask, dtype=np.uint8)
    dr = None if draw is None else np.ascontiguousarray(draw, dtype=np.int64)
    p = np.array(params, dtype=np.float64)
    fpar = None if fixed_params is None else np.ascontiguousarray(fixed_params, dtype=np.float64)
    value = ctypes.c_double()
    iters = ctypes.c_int()
    stop = ctypes.c_int()
    st = L.or_register(_ptr(fixed, ctypes.c_float), ctypes.byref(fgeo), _ptr(moving, ctypes.c_float),
                       ctypes.byref(mgeo), _ptr(fm, ctypes.c_uint8), _ptr(mm, ctypes.c_uint8),
                       _ptr(dr, ctypes.c_int64), 0 if dr is None else len(dr), bins, kind,
                       _ptr(p, ctypes.c_double), _ptr(fpar, ctypes.c_double),
                       0 if fpar is None else len(fpar), iterations, minimum_step, gradient_tolerance,
                       relaxation, learning_rate, 1 if estimate_learning_rate else 0,
                       1 if shift_scales else 0, nthreads, ctypes.byref(value), ctypes.byref(iters),
                       ctypes.byref(stop))
    if st:
        raise OracleError(st)
    return {"params": p, "value": value.value, "iterations": iters.value, "stop_reason": stop.value}


def _pyr_bind():
    L = lib()
    if getattr(L, "_pyr_typed", False):
        return L
    P = ctypes.POINTER
    gp = P(OrGeometry)
    L.or_recursive_gaussian.argtypes = [P(ctypes.c_float), gp, P(ctypes.c_double), P(ctypes.c_float)]
    L.or_recursive_gaussian.restype = ctypes.c_int
    L.or_shrink_geometry.argtypes = [gp, P(ctypes.c_int64), gp]
    L.or_shrink_geometry.restype = ctypes.c_int
    L.or_resample_linear.argtypes = [P(ctypes.c_float), gp, gp, ctypes.c_double, P(ctypes.c_float)]
    L.or_resample_linear.restype = ctypes.c_int
    L._pyr_typed = True
    return L


def recursive_gaussian(volume, geo, sigma3):
    """Zero-order recursive Gaussian (filters/recursive_gaussian.rs), physical sigma per axis."""
    L = _pyr_bind()
    v = np.ascontiguousarray(volume, dtype=np.float32)
    s = np.ascontiguousarray(sigma3, dtype=np.float64)
    out = np.empty_like(v)
    st = L.or_recursive_gaussian(_ptr(v, ctypes.c_float), ctypes.byref(geo), _ptr(s, ctypes.c_double),
                                 _ptr(out, ctypes.c_float))
    if st:
        raise OracleError(st)
    return out


def shrink_geometry(geo, factors):
    """ShrinkImageFilter output grid (filters/shrink.rs:51-95)."""
    L = _pyr_bind()
    f = np.ascontiguousarray(factors, dtype=np.int64)
    out = OrGeometry()
    st = L.or_shrink_geometry(ctypes.byref(geo), _ptr(f, ctypes.c_int64), ctypes.byref(out))
    if st:
        raise OracleError(st)
    return out


def resample_linear(volume, geo_in, geo_out, fill=0.0):
    """ResampleImageFilter through the identity, linear (transform/resample.rs:226-290)."""
    L = _pyr_bind()
    v = np.ascontiguousarray(volume, dtype=np.float32)
    n = int(geo_out.size[0] * geo_out.size[1] * geo_out.size[2])
    out = np.empty(n, dtype=np.float32)
    st = L.or_resample_linear(_ptr(v, ctypes.c_float), ctypes.byref(geo_in), ctypes.byref(geo_out), float(fill),
                              _ptr(out, ctypes.c_float))
    if st:
        raise OracleError(st)
    return out.reshape(int(geo_out.size[2]), int(geo_out.size[1]), int(geo_out.size[0]))


def resample_nearest(volume, geo_in, geo_out, fill=0.0):
    """ResampleImageFilter through the identity, nearest neighbour (interpolator.rs:36-54)."""
    L = _pyr_bind()
    if not hasattr(L.or_resample_nearest, "_typed"):
        L.or_resample_nearest.argtypes = L.or_resample_linear.argtypes
        L.or_resample_nearest.restype = ctypes.c_int
        L.or_resample_nearest._typed = True
    v = np.ascontiguousarray(volume, dtype=np.float32)
    n = int(geo_out.size[0] * geo_out.size[1] * geo_out.size[2])
    out = np.empty(n, dtype=np.float32)
    st = L.or_resample_nearest(_ptr(v, ctypes.c_float), ctypes.byref(geo_in), ctypes.byref(geo_out), float(fill),
                               _ptr(out, ctypes.c_float))
    if st:
        raise OracleError(st)
    return out.reshape(int(geo_out.size[2]), int(geo_out.size[1]), int(geo_out.size[0]))


def level_mask(mask, geo, level_geo):
    """level_mask_on_device without virtual domain or fixed-initial transform
    (registration/method.rs:3068-3110): the user mask resampled nearest-neighbour onto
    the level's grid, fill 0, nonzero = inside."""
    return (resample_nearest(np.asarray(mask, dtype=np.float32), geo, level_geo, 0.0) != 0).astype(np.uint8)


def pyramid_level(fixed, fgeo, moving, mgeo, sigma, factors, sigma_physical=True):
    """prepare_level (registration/method.rs:2416) without virtual domain, fixed-initial
    transform or masks: returns (fixed_level, fixed_level_geo, moving_level)."""
    s3 = [sigma if sigma_physical else sigma * fgeo.spacing[d] for d in range(3)]
    smooth = any(v != 0.0 for v in s3)
    sf = recursive_gaussian(fixed, fgeo, s3) if smooth else np.ascontiguousarray(fixed, dtype=np.float32)
    sm = recursive_gaussian(moving, mgeo, s3) if smooth else np.ascontiguousarray(moving, dtype=np.float32)
    if all(int(f) == 1 for f in factors):
        return sf, fgeo, sm
    cg = shrink_geometry(fgeo, factors)
    return resample_linear(sf, fgeo, cg, 0.0), cg, sm
