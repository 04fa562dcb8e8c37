"""Registration driver over the device metric (the reference's kept callers).

`register_rsgd` is one level of `ImageRegistrationMethod` as the reference drives
its device metric (registration/method.rs:3140-3400): regular-step gradient descent
(optimizer.rs:271-440) with physical-shift scales and a once-estimated learning rate
(scales.rs:572-871, `set_optimizer_as_regular_step_gradient_descent_estimated` +
`set_optimizer_scales_from_physical_shift`). `centered_initialize` is
CenteredTransformInitializer in Geometry mode (initializer.rs:56-105). The loop runs
in the library (csrc/register.cpp); every objective call is the device metric.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from .metric import DeviceImage, DeviceMattesMetric
from .transforms import ParametricTransform

STOP_REASONS = {0: "MaxIterations", 1: "StepTooSmall", 2: "Converged", 3: "GradientConverged"}


class MiRsgdConfig(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("minimum_step", ctypes.c_double),
                ("gradient_tolerance", ctypes.c_double), ("relaxation", ctypes.c_double),
                ("learning_rate", ctypes.c_double), ("estimate_learning_rate", ctypes.c_int),
                ("physical_shift_scales", ctypes.c_int), ("trace", ctypes.POINTER(ctypes.c_double)),
                ("trace_rows", ctypes.c_int)]


class MiRsgdResult(ctypes.Structure):
    _fields_ = [("value", ctypes.c_double), ("valid", ctypes.c_int64), ("iterations", ctypes.c_int),
                ("stop_reason", ctypes.c_int), ("evaluations", ctypes.c_int)]


@dataclass
class LevelResult:
    """registration/method.rs:728-800 (per level)."""
    value: float
    iterations: int
    stop_reason: str
    valid_points: int
    evaluations: int
    trace: np.ndarray | None = None  # rows [value, params, derivative] per evaluation


def _bind():
    L = _lib.load()
    if getattr(L, "_rsgd_bound", False):
        return L
    P = ctypes.POINTER
    L.mi_register_rsgd.argtypes = [ctypes.c_void_p, ctypes.c_int, P(ctypes.c_double), ctypes.c_int,
                                   P(MiRsgdConfig), P(ctypes.c_double), ctypes.c_int, P(MiRsgdResult)]
    L.mi_register_rsgd.restype = ctypes.c_int
    L.mi_centered_initialize.argtypes = [P(_lib.MiGeometry), P(_lib.MiGeometry), P(ctypes.c_double),
                                         P(ctypes.c_double)]
    L.mi_centered_initialize.restype = ctypes.c_int
    L._rsgd_bound = True
    return L


def centered_initialize(fixed: DeviceImage, moving: DeviceImage):
    """(center, translation) of CenteredTransformInitializer(Geometry)."""
    L = _bind()
    c = np.zeros(3)
    t = np.zeros(3)
    dp = ctypes.POINTER(ctypes.c_double)
    _lib.check(L.mi_centered_initialize(ctypes.byref(fixed.geo), ctypes.byref(moving.geo),
                                        c.ctypes.data_as(dp), t.ctypes.data_as(dp)))
    return c, t


def register_rsgd(metric: DeviceMattesMetric, transform: ParametricTransform, iterations: int = 100,
                  minimum_step: float = 1e-4, gradient_tolerance: float = 1e-4, relaxation: float = 0.5,
                  learning_rate: float | None = None, physical_shift_scales: bool = True,
                  record: bool = False) -> LevelResult:
    """Optimise `transform` in place (its parameters are updated). With `record`, the
    result carries every evaluation's value, parameters and derivative."""
    L = _bind()
    p = np.ascontiguousarray(transform.params, dtype=np.float64).copy()
    rows = int(iterations) + 1 if record else 0
    trace = np.zeros((rows, 1 + 2 * p.size)) if record else None
    cfg = MiRsgdConfig(int(iterations), float(minimum_step), float(gradient_tolerance), float(relaxation),
                       1.0 if learning_rate is None else float(learning_rate),
                       1 if learning_rate is None else 0, 1 if physical_shift_scales else 0,
                       trace.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if record else None, rows)
    fp = np.ascontiguousarray(transform.fixed_params, dtype=np.float64)
    res = MiRsgdResult()
    dp = ctypes.POINTER(ctypes.c_double)
    _lib.check(L.mi_register_rsgd(metric.handle, transform.kind, fp.ctypes.data_as(dp) if fp.size else None,
                                  fp.size, ctypes.byref(cfg), p.ctypes.data_as(dp), p.size, ctypes.byref(res)),
               metric.ctx.handle)
    transform.set_parameters(p)
    return LevelResult(res.value, res.iterations, STOP_REASONS.get(res.stop_reason, str(res.stop_reason)),
                       res.valid, res.evaluations, None if trace is None else trace[:res.evaluations])


@dataclass
class MultiLevelResult:
    """RegistrationResult::from_levels (registration/method.rs): the final parameters
    and one record per level, coarsest first."""
    params: np.ndarray
    levels: list


def register_multilevel(fixed: DeviceImage, moving: DeviceImage, transform: ParametricTransform,
                        shrink_factors=(4, 2, 1), smoothing_sigmas=(2.0, 1.0, 0.0), sigmas_physical: bool = True,
                        bins: int = 32, strategy: int | None = 2, percentage: float = 0.1, seed: int = 0,
                        iterations: int = 200, fixed_mask: DeviceImage | None = None, **rsgd) -> MultiLevelResult:
    """The device registration loop of ImageRegistrationMethod::execute_on_device
    (registration/method.rs:2698-2880) for the Mattes metric: per level, the
    pyramid level (prepare_level: smoothed fixed resampled onto its shrunk grid,
    smoothed moving), the level's fixed mask (level_mask_on_device, method.rs:3068-
    3110: the user mask resampled nearest-neighbour onto the level's grid, fill 0),
    the level's sample draw (same strategy, percentage and seed, over the level's
    fixed grid, then gated by the mask), then one regular-step gradient descent run
    from the previous level's parameters. `transform` is updated in place."""
    from .metric import pyramid_level
    if len(shrink_factors) != len(smoothing_sigmas):
        raise ValueError("PyramidScheduleLength: shrink and smoothing schedules differ in length")
    if fixed_mask is not None and tuple(fixed_mask.size) != tuple(fixed.size):
        raise ValueError("MaskSizeMismatch: the fixed mask must lie on the fixed image's grid")
    records = []
    for f, s in zip(shrink_factors, smoothing_sigmas):
        fl, ml = pyramid_level(fixed, moving, s, f, sigmas_physical)
        lm = None if fixed_mask is None else fixed_mask.resample_nearest(fl.geo, 0.0)
        metric = DeviceMattesMetric.from_device_sampled(fl, ml, fixed_mask=lm, bins=bins, strategy=strategy,
                                                        percentage=percentage, seed=seed)
        fl.free()
        ml.free()
        if lm is not None:
            lm.free()
        records.append(register_rsgd(metric, transform, iterations=iterations, **rsgd))
        metric.close()
    return MultiLevelResult(np.array(transform.params, dtype=np.float64), records)


class BatchRegistration:
    """Many registrations of uneven sizes advanced together on the device (mi_batch_*):
    one pass of histogram, derivative and optimizer-step launches per iteration for
    every still-active pair, replayed from a CUDA graph until all pairs have stopped.
    Affine (centres given per pair) or translation family; one bin count, one
    sampling rule per pair."""

    def __init__(self, fixed_images, moving_images, bins: int = 50, kind: int = 0, centers=None,
                 strategy: int | None = None, percentage: float = 1.0, seeds=None):
        from .metric import SAMPLING_NONE
        L = _lib.load()
        if not getattr(L, "_batch_bound", False):
            P = ctypes.POINTER
            vp = ctypes.c_void_p
            L.mi_batch_create.argtypes = [vp, ctypes.c_int, P(vp), P(vp), P(_lib.MiSampling), ctypes.c_int,
                                          ctypes.c_int, P(ctypes.c_double), ctypes.c_int, P(vp)]
            L.mi_batch_register.argtypes = [vp, P(MiRsgdConfig), ctypes.c_int, P(ctypes.c_double), P(MiRsgdResult)]
            L.mi_batch_shape.argtypes = [vp, P(ctypes.c_int), P(ctypes.c_int), P(ctypes.c_int)]
            L.mi_batch_destroy.argtypes = [vp]
            for f in ("mi_batch_create", "mi_batch_register", "mi_batch_shape", "mi_batch_destroy"):
                getattr(L, f).restype = ctypes.c_int
            L._batch_bound = True
        n = len(fixed_images)
        if len(moving_images) != n:
            raise ValueError("one moving image per fixed image")
        self.n = n
        self.kind = kind
        self.nparams = {0: 12, 3: 3}.get(kind)
        if self.nparams is None:
            raise ValueError("the batched form takes affine (0) or translation (3)")
        self.ctx = fixed_images[0].ctx
        fx = (ctypes.c_void_p * n)(*[f.handle for f in fixed_images])
        mv = (ctypes.c_void_p * n)(*[m.handle for m in moving_images])
        smp = None
        if strategy is not None and strategy != SAMPLING_NONE:
            seeds = seeds if seeds is not None else [0] * n
            smp = (_lib.MiSampling * n)(*[_lib.MiSampling(strategy, float(percentage), int(s) & (2**64 - 1), None, 0)
                                          for s in seeds])
        fp = None
        nfixed = 0
        if kind == 0:
            c = np.ascontiguousarray(centers, dtype=np.float64).reshape(n, 3)
            self._centers = c
            fp = c.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            nfixed = 3
        h = ctypes.c_void_p()
        _lib.check(L.mi_batch_create(self.ctx.handle, n, fx, mv, smp, int(bins), kind, fp, nfixed, ctypes.byref(h)),
                   self.ctx.handle)
        self.handle = h

    def register(self, params, iterations: int = 100, minimum_step: float = 1e-4, gradient_tolerance: float = 1e-4,
                 relaxation: float = 0.5, learning_rate: float | None = None, physical_shift_scales: bool = True,
                 autotune: bool = True):
        """Runs every pair from `params` (n × nparams); returns (params, [LevelResult])."""
        p = np.ascontiguousarray(params, dtype=np.float64).reshape(self.n, self.nparams).copy()
        cfg = MiRsgdConfig(int(iterations), float(minimum_step), float(gradient_tolerance), float(relaxation),
                           1.0 if learning_rate is None else float(learning_rate),
                           1 if learning_rate is None else 0, 1 if physical_shift_scales else 0, None, 0)
        res = (MiRsgdResult * self.n)()
        _lib.check(_lib.load().mi_batch_register(self.handle, ctypes.byref(cfg), 1 if autotune else 0,
                                                 p.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), res),
                   self.ctx.handle)
        out = [LevelResult(r.value, r.iterations, STOP_REASONS.get(r.stop_reason, str(r.stop_reason)), r.valid,
                           r.evaluations) for r in res]
        return p, out

    def pair_seconds(self) -> np.ndarray:
        """Per pair, the device-timed interval from the start of the last register() run
        to the optimizer step at which the pair stopped (mi_batch_pair_seconds)."""
        out = np.zeros(self.n)
        L = _lib.load()
        L.mi_batch_pair_seconds.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int]
        L.mi_batch_pair_seconds.restype = ctypes.c_int
        _lib.check(L.mi_batch_pair_seconds(self.handle, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), self.n),
                   self.ctx.handle)
        return out

    def shape(self):
        """(chunk size, histogram copies, chunk count) in use."""
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.check(_lib.load().mi_batch_shape(self.handle, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def close(self):
        if getattr(self, "handle", None):
            _lib.load().mi_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
