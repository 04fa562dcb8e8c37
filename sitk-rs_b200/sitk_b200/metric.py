"""Host-side mirror of the reference's device metric seam.

`DeviceImage` follows crates/sitk/src/cuda/image.rs (upload of any scalar pixel type
to a device f32 volume, to_host), and `DeviceMattesMetric` follows
registration/device.rs:632-800 (from_device, from_device_sampled, value, evaluate),
returning a `MetricValue` (registration/metric.rs:1021-1030). Everything runs through
the C ABI of libmi_b200.so; there is no other compute path.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

from . import _lib
from .transforms import ParametricTransform

_DTYPES = {np.dtype(np.uint8): 0, np.dtype(np.int8): 1, np.dtype(np.uint16): 2,
           np.dtype(np.int16): 3, np.dtype(np.uint32): 4, np.dtype(np.int32): 5,
           np.dtype(np.uint64): 6, np.dtype(np.int64): 7, np.dtype(np.float32): 8,
           np.dtype(np.float64): 9}

SAMPLING_NONE, SAMPLING_REGULAR, SAMPLING_RANDOM, SAMPLING_EXPLICIT = 0, 1, 2, 3


def geometry(size, spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0),
             direction=(1, 0, 0, 0, 1, 0, 0, 0, 1)) -> _lib.MiGeometry:
    g = _lib.MiGeometry()
    for i in range(3):
        g.size[i] = int(size[i])
        g.spacing[i] = float(spacing[i])
        g.origin[i] = float(origin[i])
    for i in range(9):
        g.direction[i] = float(np.asarray(direction, dtype=np.float64).ravel()[i])
    return g


class Context:
    """One device, one stream (cuda/backend.rs:30-160)."""

    def __init__(self, device: int = 0):
        L = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(L.mi_context_create(device, ctypes.byref(h)))
        self.handle = h
        self.device = device

    def sync(self):
        _lib.check(_lib.load().mi_context_sync(self.handle), self.handle)

    def stream(self) -> int:
        return _lib.load().mi_context_stream(self.handle) or 0

    def close(self):
        if self.handle:
            _lib.load().mi_context_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Context | None = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


class DeviceImage:
    """A 3-D scalar volume resident on the device as f32 (x-fastest).

    `array` is indexed [z, y, x] (numpy C order of an x-fastest buffer)."""

    def __init__(self, handle, ctx: Context, geo: _lib.MiGeometry):
        self.handle = handle
        self.ctx = ctx
        self.geo = geo

    @classmethod
    def upload(cls, array, spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0),
               direction=(1, 0, 0, 0, 1, 0, 0, 0, 1), ctx: Context | None = None) -> "DeviceImage":
        ctx = ctx or default_context()
        a = np.ascontiguousarray(array)
        if a.ndim != 3:
            raise ValueError("the device metric is 3-D only")  # NotThreeDimensional
        if np.iscomplexobj(a):
            code = 100
        else:
            code = _DTYPES.get(a.dtype)
            if code is None:
                raise TypeError(f"unsupported pixel type {a.dtype}")
        geo = geometry((a.shape[2], a.shape[1], a.shape[0]), spacing, origin, direction)
        h = ctypes.c_void_p()
        _lib.check(_lib.load().mi_image_upload(ctx.handle, a.ctypes.data_as(ctypes.c_void_p), code,
                                               ctypes.byref(geo), ctypes.byref(h)), ctx.handle)
        return cls(h, ctx, geo)

    @classmethod
    def read(cls, path: str, ctx: "Context | None" = None) -> "DeviceImage":
        """A MetaImage (.mha / .mhd, mi_image_read_meta) or NIfTI-1 (.nii, .hdr / .img,
        optionally .gz, mi_image_read_nifti) file read and uploaded, by its extension."""
        ctx = ctx or default_context()
        h = ctypes.c_void_p()
        if _is_nifti_name(path):
            _lib.check(_nifti_lib().mi_image_read_nifti(ctx.handle, os.fsencode(path), ctypes.byref(h)), ctx.handle)
        else:
            _lib.check(_lib.load().mi_image_read_meta(ctx.handle, os.fsencode(path), ctypes.byref(h)), ctx.handle)
        geo = _lib.MiGeometry()
        _lib.check(_lib.load().mi_image_geometry(h, ctypes.byref(geo)))
        return cls(h, ctx, geo)

    @classmethod
    def from_device_ptr(cls, ptr: int, size, spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0),
                        direction=(1, 0, 0, 0, 1, 0, 0, 0, 1), ctx: Context | None = None):
        ctx = ctx or default_context()
        geo = geometry(size, spacing, origin, direction)
        h = ctypes.c_void_p()
        _lib.check(_lib.load().mi_image_from_device(ctx.handle, ctypes.c_void_p(ptr), ctypes.byref(geo),
                                                    ctypes.byref(h)), ctx.handle)
        return cls(h, ctx, geo)

    @property
    def size(self):
        return tuple(int(self.geo.size[i]) for i in range(3))

    def to_host(self) -> np.ndarray:
        nx, ny, nz = self.size
        out = np.empty((nz, ny, nx), dtype=np.float32)
        _lib.check(_lib.load().mi_image_to_host(self.handle, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                out.size), self.ctx.handle)
        return out

    def device_ptr(self) -> int:
        return _lib.load().mi_image_device_ptr(self.handle) or 0

    def smooth(self, sigma) -> "DeviceImage":
        """Zero-order recursive Gaussian (filters/recursive_gaussian.rs); `sigma` is a
        physical sigma per axis (or one for all)."""
        s = np.broadcast_to(np.asarray(sigma, dtype=np.float64), (3,)).copy()
        h = ctypes.c_void_p()
        _lib.check(_lib.load().mi_image_smooth(self.ctx.handle, self.handle,
                                               s.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(h)),
                   self.ctx.handle)
        return DeviceImage(h, self.ctx, _copy_geo(self.geo))

    def resample(self, grid: _lib.MiGeometry, fill: float = 0.0) -> "DeviceImage":
        """Linear resampling onto `grid` through the identity (transform/resample.rs)."""
        h = ctypes.c_void_p()
        _lib.check(_lib.load().mi_image_resample(self.ctx.handle, self.handle, ctypes.byref(grid), float(fill),
                                                 ctypes.byref(h)), self.ctx.handle)
        return DeviceImage(h, self.ctx, _copy_geo(grid))

    def resample_nearest(self, grid: _lib.MiGeometry, fill: float = 0.0) -> "DeviceImage":
        """Nearest-neighbour resampling onto `grid` through the identity
        (transform/interpolator.rs:36-54), as level masks are formed."""
        h = ctypes.c_void_p()
        _lib.check(_lib.load().mi_image_resample_nearest(self.ctx.handle, self.handle, ctypes.byref(grid),
                                                         float(fill), ctypes.byref(h)), self.ctx.handle)
        return DeviceImage(h, self.ctx, _copy_geo(grid))

    def free(self):
        if self.handle:
            _lib.load().mi_image_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


@dataclass
class MetricValue:
    """registration/metric.rs:1021-1030."""
    value: float
    derivative: np.ndarray
    valid_points: int


class DeviceMattesMetric:
    """Mattes MI over two device-resident images (registration/device.rs:632-800)."""

    def __init__(self, handle, ctx: Context):
        self.handle = handle
        self.ctx = ctx
        # argument buffers reused by every evaluate() call: building numpy ctypes views
        # per call costs several microseconds, a sizeable share of a ~70 µs evaluation
        n = 12
        self._p = (ctypes.c_double * n)()
        self._fp = (ctypes.c_double * n)()
        self._d = (ctypes.c_double * n)()
        self._v = ctypes.c_double()
        self._n = ctypes.c_int64()
        self._vref = ctypes.byref(self._v)
        self._nref = ctypes.byref(self._n)
        # numpy views over the same buffers: parameters in and the derivative out without
        # building Python lists
        self._pnp = np.frombuffer(self._p, dtype=np.float64)
        self._fpnp = np.frombuffer(self._fp, dtype=np.float64)
        self._dnp = np.frombuffer(self._d, dtype=np.float64)
        self._fn = _lib.load_raw().mi_metric_value_and_derivative

    @classmethod
    def from_device(cls, fixed: DeviceImage, moving: DeviceImage, bins: int = 50):
        return cls.from_device_sampled(fixed, moving, None, None, None, bins)

    @classmethod
    def from_device_sampled(cls, fixed: DeviceImage, moving: DeviceImage, fixed_mask=None,
                            moving_mask=None, samples=None, bins: int = 50, *,
                            strategy: int | None = None, percentage: float = 1.0, seed: int = 0,
                            moving_storage: str = "f32", texture: str = "auto",
                            _metric: int = _lib.METRIC_MATTES):
        """`samples` is an explicit flat-index list (FixedSamples::selected_indices);
        alternatively `strategy`/`percentage`/`seed` draw on the device exactly as
        draw_samples does (registration/metric.rs:419-437). `moving_storage` "bf16"
        keeps the moving volume rounded to BF16 (mi_metric_create_ex). `texture` "3d"
        keeps the moving volume in a 3-D texture instead of the layered one (same
        results; MI_TEXTURE_3D)."""
        storage = {"f32": 0, "bf16": 1}.get(moving_storage)
        if storage is None:
            raise ValueError("moving_storage is 'f32' or 'bf16'")
        tex = {"auto": 0, "3d": 1}.get(texture)
        if tex is None:
            raise ValueError("texture is 'auto' or '3d'")
        ctx = fixed.ctx
        smp = None
        keep = []
        if samples is not None:
            idx = np.ascontiguousarray(samples, dtype=np.int64)
            keep.append(idx)
            smp = _lib.MiSampling(SAMPLING_EXPLICIT, 1.0, 0,
                                  idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), idx.size)
        elif strategy is not None and strategy != SAMPLING_NONE:
            smp = _lib.MiSampling(strategy, float(percentage), int(seed) & (2**64 - 1), None, 0)
        mm = None
        if moving_mask is not None:
            mm = np.ascontiguousarray(np.asarray(moving_mask) != 0, dtype=np.uint8)
            keep.append(mm)
        fm_handle = None
        if fixed_mask is not None:
            fm_handle = fixed_mask.handle if isinstance(fixed_mask, DeviceImage) else None
            if fm_handle is None:
                fmi = DeviceImage.upload(np.asarray(fixed_mask, dtype=np.float32), ctx=ctx)
                keep.append(fmi)
                fm_handle = fmi.handle
        h = ctypes.c_void_p()
        opts = _lib.MiMetricOptions(storage, int(_metric), tex)
        _lib.check(_lib.load().mi_metric_create_ex(
            ctx.handle, fixed.handle, moving.handle, fm_handle,
            None if mm is None else mm.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)),
            None if smp is None else ctypes.byref(smp), int(bins), ctypes.byref(opts), ctypes.byref(h)), ctx.handle)
        return cls(h, ctx)

    def info(self) -> dict:
        inf = _lib.MiMetricInfo()
        _lib.check(_lib.load().mi_metric_info_get(self.handle, ctypes.byref(inf)), self.ctx.handle)
        return {f: getattr(inf, f) for f, _ in _lib.MiMetricInfo._fields_}

    def sample_count(self) -> int:
        return int(self.info()["n_samples"])

    def sample_order(self) -> np.ndarray:
        """Flat fixed-grid index of every sample in the order the device walks them
        (the order of per-sample outputs)."""
        n = self.sample_count()
        out = np.zeros(max(n, 1), dtype=np.uint32)
        _lib.check(_lib.load().mi_metric_sample_order(self.handle, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)),
                                                      n), self.ctx.handle)
        return out[:n]

    def value(self, transform: ParametricTransform) -> float:
        if getattr(transform, "BSPLINE", None):
            return self._bspline(transform, False).value
        st = self.stages(transform)
        v = ctypes.c_double()
        _lib.check(_lib.load().mi_metric_value(self.handle, st.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                               st.size // 12, ctypes.byref(v), None), self.ctx.handle)
        return v.value

    def value_stages(self, stages) -> tuple[float, int]:
        st = np.ascontiguousarray(stages, dtype=np.float64).ravel()
        v = ctypes.c_double()
        n = ctypes.c_int64()
        _lib.check(_lib.load().mi_metric_value(self.handle, st.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                               st.size // 12, ctypes.byref(v), ctypes.byref(n)), self.ctx.handle)
        return v.value, n.value

    def _bspline(self, transform, derivative: bool):
        fp = np.ascontiguousarray(transform.fixed_params, dtype=np.float64)
        c = np.ascontiguousarray(transform.params, dtype=np.float64)
        d = np.zeros(c.size) if derivative else None
        v = ctypes.c_double()
        n = ctypes.c_int64()
        dp = ctypes.POINTER(ctypes.c_double)
        _lib.check(_lib.load().mi_metric_value_and_derivative_bspline(
            self.handle, fp.ctypes.data_as(dp), c.ctypes.data_as(dp), c.size, ctypes.byref(v),
            d.ctypes.data_as(dp) if derivative else None, ctypes.byref(n)), self.ctx.handle)
        return MetricValue(v.value, d, n.value)

    def evaluate(self, transform: ParametricTransform) -> MetricValue:
        if getattr(transform, "BSPLINE", None):
            return self._bspline(transform, True)
        params, fixed = transform.params, transform.fixed_params
        n, nf = params.shape[0], fixed.shape[0]
        if n > 12 or nf > 12:
            raise ValueError("at most 12 parameters and 12 fixed parameters")
        self._pnp[:n] = params
        if nf:
            self._fpnp[:nf] = fixed
        st = self._fn(self.handle, int(transform.kind), self._p, n, self._fp if nf else None, nf, self._vref, self._d,
                      self._nref)
        if st:
            _lib.check(st, self.ctx.handle)
        return MetricValue(self._v.value, self._dnp[:n].copy(), self._n.value)

    def evaluate_stages(self, stages, jac0, jacc) -> MetricValue:
        st = np.ascontiguousarray(stages, dtype=np.float64).ravel()
        j0 = np.ascontiguousarray(jac0, dtype=np.float64).ravel()
        jc = np.ascontiguousarray(jacc, dtype=np.float64).ravel()
        P = j0.size // 3
        d = np.zeros(P)
        v = ctypes.c_double()
        n = ctypes.c_int64()
        dp = ctypes.POINTER(ctypes.c_double)
        _lib.check(_lib.load().mi_metric_value_and_derivative_stages(
            self.handle, st.ctypes.data_as(dp), st.size // 12, j0.ctypes.data_as(dp), jc.ctypes.data_as(dp),
            P, ctypes.byref(v), d.ctypes.data_as(dp), ctypes.byref(n)), self.ctx.handle)
        return MetricValue(v.value, d, n.value)

    def sample_decisions(self, stages):
        st = np.ascontiguousarray(stages, dtype=np.float64).ravel()
        n = self.sample_count()
        status = np.empty(n, dtype=np.int8)
        fb = np.empty(n, dtype=np.int32)
        mb = np.empty(n, dtype=np.int32)
        flat = np.empty(n, dtype=np.int64)
        exact = np.empty(n, dtype=np.int8)
        P = ctypes.POINTER
        _lib.check(_lib.load().mi_metric_sample_decisions(
            self.handle, st.ctypes.data_as(P(ctypes.c_double)), st.size // 12,
            status.ctypes.data_as(P(ctypes.c_int8)), fb.ctypes.data_as(P(ctypes.c_int32)),
            mb.ctypes.data_as(P(ctypes.c_int32)), flat.ctypes.data_as(P(ctypes.c_int64)),
            exact.ctypes.data_as(P(ctypes.c_int8)), n), self.ctx.handle)
        return {"status": status, "fi": fb, "mi": mb, "flat": flat, "exact": exact}

    @staticmethod
    def stages(transform: ParametricTransform) -> np.ndarray:
        """The transform's point-map stage (matrix row-major, offset), formed by the
        library's own host code for the family."""
        return transform_stage(transform)

    def close(self):
        if self.handle:
            _lib.load().mi_metric_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DeviceMeanSquaresMetric(DeviceMattesMetric):
    """registration/device.rs:203-365 DeviceMeanSquaresMetric: value = Σ(m − f)²/count
    and its parameter derivative, over the same sample set, masks and sampler as the
    Mattes metric (mi_metric_create_ex with MI_METRIC_MEAN_SQUARES)."""

    @classmethod
    def from_device(cls, fixed: DeviceImage, moving: DeviceImage):
        return cls.from_device_sampled(fixed, moving)

    @classmethod
    def from_device_sampled(cls, fixed: DeviceImage, moving: DeviceImage, fixed_mask=None, moving_mask=None,
                            samples=None, *, strategy: int | None = None, percentage: float = 1.0, seed: int = 0,
                            moving_storage: str = "f32", texture: str = "auto"):
        return super().from_device_sampled(fixed, moving, fixed_mask, moving_mask, samples, 0, strategy=strategy,
                                           percentage=percentage, seed=seed, moving_storage=moving_storage,
                                           texture=texture,
                                           _metric=_lib.METRIC_MEAN_SQUARES)


class DeviceCorrelationMetric(DeviceMattesMetric):
    """registration/device.rs:474-575 DeviceCorrelationMetric: value = −sfm²/(sff·smm)
    over the mean-subtracted samples, two device passes (means, then moments), and its
    parameter derivative (mi_metric_create_ex with MI_METRIC_CORRELATION)."""

    @classmethod
    def from_device(cls, fixed: DeviceImage, moving: DeviceImage):
        return cls.from_device_sampled(fixed, moving)

    @classmethod
    def from_device_sampled(cls, fixed: DeviceImage, moving: DeviceImage, fixed_mask=None, moving_mask=None,
                            samples=None, *, strategy: int | None = None, percentage: float = 1.0, seed: int = 0,
                            moving_storage: str = "f32", texture: str = "auto"):
        return super().from_device_sampled(fixed, moving, fixed_mask, moving_mask, samples, 0, strategy=strategy,
                                           percentage=percentage, seed=seed, moving_storage=moving_storage,
                                           texture=texture,
                                           _metric=_lib.METRIC_CORRELATION)


def transform_form(transform: ParametricTransform):
    """(stage[12], jac0[3×P], jacc[3][3×P]) from the library's host transform code
    (mi_transform_form): the matrix/offset the family multiplies and its Jacobian's
    affine form, in the reference's operation order."""
    p = np.ascontiguousarray(transform.params, dtype=np.float64)
    fp = np.ascontiguousarray(transform.fixed_params, dtype=np.float64)
    st = np.zeros(12)
    P = transform.nparams
    j0 = np.zeros(3 * P)
    jc = np.zeros(9 * P)
    dp = ctypes.POINTER(ctypes.c_double)
    _lib.check(_lib.load().mi_transform_form(transform.kind, p.ctypes.data_as(dp), p.size,
                                             fp.ctypes.data_as(dp) if fp.size else None, fp.size,
                                             st.ctypes.data_as(dp), j0.ctypes.data_as(dp),
                                             jc.ctypes.data_as(dp)))
    return st, j0.reshape(3, P), jc.reshape(3, 3, P)


def transform_stage(transform: ParametricTransform) -> np.ndarray:
    """The family's point-map stage: matrix row-major then offset."""
    return transform_form(transform)[0]


def enable_timing(metric: DeviceMattesMetric, on: bool = True, per_kernel: bool = False) -> None:
    """Record CUDA events around each evaluation (and, with per_kernel, after each of
    its kernels) for benchmark accounting."""
    mode = 0 if not on else (2 if per_kernel else 1)
    _lib.check(_lib.load().mi_metric_timing_enable(metric.handle, mode), metric.ctx.handle)


def read_timing(metric: DeviceMattesMetric) -> tuple[np.ndarray, int]:
    """Accumulated device milliseconds [evaluation, histogram, tail, derivative] and the
    evaluation count since the last read (then reset)."""
    ms = np.zeros(4)
    n = ctypes.c_int64()
    _lib.check(_lib.load().mi_metric_timing_read(metric.handle, ms.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                 ctypes.byref(n)), metric.ctx.handle)
    return ms, n.value


def set_fused(metric: DeviceMattesMetric, fused: bool) -> None:
    """Choose the launch form: one cooperative kernel (True) or two kernels (False).
    Both compute the same histogram, tail and moments."""
    _lib.check(_lib.load().mi_metric_set_fused(metric.handle, 1 if fused else 0), metric.ctx.handle)


def get_fused(metric: DeviceMattesMetric) -> bool:
    f = ctypes.c_int()
    _lib.check(_lib.load().mi_metric_get_fused(metric.handle, ctypes.byref(f)), metric.ctx.handle)
    return bool(f.value)


def set_tile_staging(metric: DeviceMattesMetric, on: bool) -> None:
    """Choose the histogram pass's corner source: TMA-staged moving tiles in shared
    memory (True) or the moving volume's texture (False, the default). Same bits."""
    _lib.check(_lib.load().mi_metric_set_tile_staging(metric.handle, 1 if on else 0), metric.ctx.handle)


def get_tile_staging(metric: DeviceMattesMetric) -> tuple[bool, int]:
    """The staged-tile setting and how many evaluations ran with staged tiles."""
    on = ctypes.c_int()
    n = ctypes.c_int64()
    _lib.check(_lib.load().mi_metric_get_tile_staging(metric.handle, ctypes.byref(on), ctypes.byref(n)),
               metric.ctx.handle)
    return bool(on.value), n.value


def _copy_geo(g: _lib.MiGeometry) -> _lib.MiGeometry:
    out = _lib.MiGeometry()
    ctypes.pointer(out)[0] = g
    return out


def shrink_geometry(geo: _lib.MiGeometry, factors) -> _lib.MiGeometry:
    """ShrinkImageFilter's output grid (filters/shrink.rs:51-95)."""
    f = np.broadcast_to(np.asarray(factors, dtype=np.int64), (3,)).copy()
    out = _lib.MiGeometry()
    _lib.check(_lib.load().mi_shrink_geometry(ctypes.byref(geo), f.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                              ctypes.byref(out)))
    return out


def pyramid_level(fixed: DeviceImage, moving: DeviceImage, sigma: float, factors, sigma_physical: bool = True):
    """One level of prepare_level (registration/method.rs:2416): (fixed_level, moving_level)."""
    f = np.broadcast_to(np.asarray(factors, dtype=np.int64), (3,)).copy()
    hf, hm = ctypes.c_void_p(), ctypes.c_void_p()
    _lib.check(_lib.load().mi_pyramid_level(fixed.ctx.handle, fixed.handle, moving.handle, float(sigma),
                                            1 if sigma_physical else 0,
                                            f.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), ctypes.byref(hf),
                                            ctypes.byref(hm)), fixed.ctx.handle)
    L = _lib.load()
    gf, gm = _lib.MiGeometry(), _lib.MiGeometry()
    _lib.check(L.mi_image_geometry(hf, ctypes.byref(gf)))
    _lib.check(L.mi_image_geometry(hm, ctypes.byref(gm)))
    return DeviceImage(hf, fixed.ctx, gf), DeviceImage(hm, moving.ctx, gm)


def _is_nifti_name(path: str) -> bool:
    p = os.fspath(path).lower()
    return p.endswith((".nii", ".nii.gz", ".hdr", ".hdr.gz", ".img", ".img.gz"))


def _nifti_lib():
    L = _lib.load()
    if not getattr(L, "_nifti_bound", False):
        L.mi_image_read_nifti.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)]
        L.mi_image_read_nifti.restype = ctypes.c_int
        L.mi_image_read_nifti_host.argtypes = [ctypes.c_char_p, ctypes.POINTER(_lib.MiGeometry),
                                               ctypes.POINTER(ctypes.c_float), ctypes.c_size_t]
        L.mi_image_read_nifti_host.restype = ctypes.c_int
        L._nifti_bound = True
    return L


def read_nifti_host(path: str):
    """A NIfTI-1 file read on the host alone (mi_image_read_nifti_host): (voxels as a
    float32 [z, y, x] array, rescaled and cast as the reader does, geometry)."""
    L = _nifti_lib()
    geo = _lib.MiGeometry()
    p = os.fsencode(path)
    _lib.check(L.mi_image_read_nifti_host(p, ctypes.byref(geo), None, 0))
    nx, ny, nz = (int(geo.size[i]) for i in range(3))
    out = np.empty((nz, ny, nx), dtype=np.float32)
    _lib.check(L.mi_image_read_nifti_host(p, ctypes.byref(geo), out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                          out.size))
    return out, geo


def read_meta_host(path: str):
    """A MetaImage file read on the host alone (mi_image_read_meta_host): (voxels as a
    float32 [z, y, x] array cast as the upload casts them, geometry)."""
    L = _lib.load()
    geo = _lib.MiGeometry()
    p = os.fsencode(path)
    _lib.check(L.mi_image_read_meta_host(p, ctypes.byref(geo), None, 0))
    nx, ny, nz = (int(geo.size[i]) for i in range(3))
    out = np.empty((nz, ny, nx), dtype=np.float32)
    _lib.check(L.mi_image_read_meta_host(p, ctypes.byref(geo), out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                         out.size))
    return out, geo
