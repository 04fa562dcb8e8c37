"""ctypes binding of libmi_b200.so (the C ABI declared in include/mi_b200.h).

The library is the only compute path: if it is missing or no CUDA device is present,
calls raise instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes
import os

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libmi_b200.so")

MI_OK = 0
STATUS_NAMES = {
    0: "MI_OK", 1: "MI_ERR_INVALID_ARGUMENT", 2: "MI_ERR_NO_DEVICE", 3: "MI_ERR_CUDA",
    4: "MI_ERR_OUT_OF_MEMORY", 5: "MI_ERR_UNSUPPORTED_PIXEL_TYPE", 6: "MI_ERR_SINGULAR_DIRECTION",
    7: "MI_ERR_TOO_FEW_HISTOGRAM_BINS", 8: "MI_ERR_CONSTANT_FIXED", 9: "MI_ERR_CONSTANT_MOVING",
    10: "MI_ERR_SAMPLE_INDEX_OUT_OF_GRID", 11: "MI_ERR_MASK_SIZE_MISMATCH",
    12: "MI_ERR_NON_AFFINE_TRANSFORM", 13: "MI_ERR_POINT_MAP_STAGE_COUNT",
    14: "MI_ERR_TOO_MANY_HISTOGRAM_BINS", 15: "MI_ERR_TIMEOUT", 16: "MI_ERR_NOT_CONVERGED",
}

# Every symbol include/mi_b200.h declares; tests check the library exports all of them.
EXPORTED = [
    "mi_status_string", "mi_context_create", "mi_context_destroy", "mi_context_sync",
    "mi_last_error", "mi_context_stream", "mi_image_upload", "mi_image_from_device",
    "mi_image_to_host", "mi_image_geometry", "mi_image_device_ptr", "mi_image_free",
    "mi_metric_create", "mi_metric_info_get", "mi_metric_sample_order", "mi_metric_destroy", "mi_metric_value",
    "mi_metric_value_and_derivative", "mi_metric_value_and_derivative_stages",
    "mi_metric_sample_decisions", "mi_transform_form", "mi_metric_timing_enable",
    "mi_metric_timing_read", "mi_metric_value_noalloc", "mi_register_rsgd",
    "mi_centered_initialize", "mi_metric_set_fused", "mi_metric_get_fused", "mi_image_smooth",
    "mi_shrink_geometry", "mi_image_resample", "mi_pyramid_level", "mi_batch_create", "mi_batch_register",
    "mi_batch_shape", "mi_batch_pair_seconds", "mi_batch_destroy", "mi_synth_pair", "mi_gemm_bf16_tn", "mi_initnet_create",
    "mi_initnet_destroy", "mi_initnet_get", "mi_initnet_set", "mi_initnet_forward", "mi_initnet_train_step",
    "mi_initnet_prepare", "mi_metric_create_ex", "mi_image_resample_nearest",
    "mi_metric_value_and_derivative_bspline", "mi_metric_bspline_records", "mi_image_read_meta",
    "mi_image_read_meta_host", "mi_image_read_nifti", "mi_image_read_nifti_host",
    "mi_metric_set_tile_staging", "mi_metric_get_tile_staging",
]


class MiGeometry(ctypes.Structure):
    _fields_ = [("size", ctypes.c_int64 * 3), ("spacing", ctypes.c_double * 3),
                ("origin", ctypes.c_double * 3), ("direction", ctypes.c_double * 9)]


class MiSampling(ctypes.Structure):
    _fields_ = [("strategy", ctypes.c_int), ("percentage", ctypes.c_double),
                ("seed", ctypes.c_uint64), ("indices", ctypes.POINTER(ctypes.c_int64)),
                ("n_indices", ctypes.c_int64)]


class MiMetricInfo(ctypes.Structure):
    _fields_ = [("bins", ctypes.c_int), ("n_samples", ctypes.c_int64),
                ("fixed_min", ctypes.c_double), ("fixed_max", ctypes.c_double),
                ("moving_min", ctypes.c_double), ("moving_max", ctypes.c_double),
                ("fixed_bin_size", ctypes.c_double), ("moving_bin_size", ctypes.c_double),
                ("fixed_normalized_min", ctypes.c_double),
                ("moving_normalized_min", ctypes.c_double)]


class MiMetricOptions(ctypes.Structure):
    _fields_ = [("moving_storage", ctypes.c_int), ("metric", ctypes.c_int), ("texture", ctypes.c_int)]


METRIC_MATTES, METRIC_MEAN_SQUARES, METRIC_CORRELATION = 0, 1, 2


class MiError(RuntimeError):
    """A named refusal from the library (mirrors DeviceMetricError / CudaError)."""

    def __init__(self, status: int, detail: str = ""):
        self.status = status
        self.name = STATUS_NAMES.get(status, str(status))
        super().__init__(f"{self.name}: {detail}" if detail else self.name)


_lib = None


def load(path: str | None = None):
    """Load the library (once). Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"{p} is missing: build it with `python sitk-rs_b200/build.py` "
                           "(there is no non-CUDA path)")
    L = ctypes.CDLL(p)
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    dp, i64p = P(ctypes.c_double), P(ctypes.c_int64)
    L.mi_status_string.argtypes = [ctypes.c_int]
    L.mi_status_string.restype = ctypes.c_char_p
    L.mi_context_create.argtypes = [ctypes.c_int, P(vp)]
    L.mi_context_destroy.argtypes = [vp]
    L.mi_context_sync.argtypes = [vp]
    L.mi_last_error.argtypes = [vp]
    L.mi_last_error.restype = ctypes.c_char_p
    L.mi_context_stream.argtypes = [vp]
    L.mi_context_stream.restype = vp
    L.mi_image_upload.argtypes = [vp, vp, ctypes.c_int, P(MiGeometry), P(vp)]
    L.mi_image_from_device.argtypes = [vp, vp, P(MiGeometry), P(vp)]
    L.mi_image_to_host.argtypes = [vp, P(ctypes.c_float), ctypes.c_size_t]
    L.mi_image_geometry.argtypes = [vp, P(MiGeometry)]
    L.mi_image_device_ptr.argtypes = [vp]
    L.mi_image_device_ptr.restype = vp
    L.mi_image_free.argtypes = [vp]
    L.mi_metric_create.argtypes = [vp, vp, vp, vp, P(ctypes.c_uint8), P(MiSampling), ctypes.c_int, P(vp)]
    L.mi_metric_create_ex.argtypes = [vp, vp, vp, vp, P(ctypes.c_uint8), P(MiSampling), ctypes.c_int,
                                      P(MiMetricOptions), P(vp)]
    L.mi_metric_create_ex.restype = ctypes.c_int
    L.mi_metric_info_get.argtypes = [vp, P(MiMetricInfo)]
    L.mi_metric_sample_order.argtypes = [vp, P(ctypes.c_uint32), ctypes.c_int64]
    L.mi_metric_sample_order.restype = ctypes.c_int
    L.mi_metric_destroy.argtypes = [vp]
    L.mi_metric_value.argtypes = [vp, dp, ctypes.c_int, dp, i64p]
    L.mi_metric_value_and_derivative.argtypes = [vp, ctypes.c_int, dp, ctypes.c_int, dp, ctypes.c_int,
                                                 dp, dp, i64p]
    L.mi_metric_value_and_derivative_stages.argtypes = [vp, dp, ctypes.c_int, dp, dp, ctypes.c_int,
                                                        dp, dp, i64p]
    L.mi_metric_sample_decisions.argtypes = [vp, dp, ctypes.c_int, P(ctypes.c_int8), P(ctypes.c_int32),
                                             P(ctypes.c_int32), i64p, P(ctypes.c_int8), ctypes.c_int64]
    L.mi_transform_form.argtypes = [ctypes.c_int, dp, ctypes.c_int, dp, ctypes.c_int, dp, dp, dp]
    L.mi_metric_value_noalloc.argtypes = [vp, vp, P(MiGeometry), vp, P(MiGeometry), vp, ctypes.c_int64,
                                          P(MiMetricInfo), dp, ctypes.c_int, vp]
    L.mi_metric_value_noalloc.restype = ctypes.c_int
    L.mi_metric_timing_enable.argtypes = [vp, ctypes.c_int]
    L.mi_metric_timing_read.argtypes = [vp, dp, i64p]
    L.mi_metric_set_fused.argtypes = [vp, ctypes.c_int]
    L.mi_image_smooth.argtypes = [vp, vp, dp, P(vp)]
    L.mi_shrink_geometry.argtypes = [P(MiGeometry), i64p, P(MiGeometry)]
    L.mi_image_resample.argtypes = [vp, vp, P(MiGeometry), ctypes.c_double, P(vp)]
    L.mi_image_resample_nearest.argtypes = [vp, vp, P(MiGeometry), ctypes.c_double, P(vp)]
    L.mi_image_resample_nearest.restype = ctypes.c_int
    L.mi_metric_value_and_derivative_bspline.argtypes = [vp, dp, dp, ctypes.c_int64, dp, dp, i64p]
    L.mi_metric_value_and_derivative_bspline.restype = ctypes.c_int
    L.mi_metric_bspline_records.argtypes = [vp, dp, dp, ctypes.c_int64, P(ctypes.c_uint16), ctypes.c_int64]
    L.mi_metric_bspline_records.restype = ctypes.c_int
    L.mi_image_read_meta.argtypes = [vp, ctypes.c_char_p, P(vp)]
    L.mi_image_read_meta.restype = ctypes.c_int
    L.mi_image_read_meta_host.argtypes = [ctypes.c_char_p, P(MiGeometry), P(ctypes.c_float), ctypes.c_size_t]
    L.mi_image_read_meta_host.restype = ctypes.c_int
    L.mi_pyramid_level.argtypes = [vp, vp, vp, ctypes.c_double, ctypes.c_int, i64p, P(vp), P(vp)]
    L.mi_metric_get_fused.argtypes = [vp, P(ctypes.c_int)]
    L.mi_metric_set_tile_staging.argtypes = [vp, ctypes.c_int]
    L.mi_metric_set_tile_staging.restype = ctypes.c_int
    L.mi_metric_get_tile_staging.argtypes = [vp, P(ctypes.c_int), i64p]
    L.mi_metric_get_tile_staging.restype = ctypes.c_int
    for name in ["mi_image_smooth", "mi_shrink_geometry", "mi_image_resample", "mi_pyramid_level",
                 "mi_metric_set_fused", "mi_metric_get_fused", "mi_metric_timing_enable", "mi_metric_timing_read", "mi_transform_form", "mi_context_create", "mi_context_destroy", "mi_context_sync", "mi_image_upload",
                 "mi_image_from_device", "mi_image_to_host", "mi_image_geometry", "mi_image_free",
                 "mi_metric_create", "mi_metric_info_get", "mi_metric_destroy", "mi_metric_value",
                 "mi_metric_value_and_derivative", "mi_metric_value_and_derivative_stages",
                 "mi_metric_sample_decisions"]:
        getattr(L, name).restype = ctypes.c_int
    _lib = L
    return L


_raw = None


def load_raw():
    """The same library through a second handle whose functions carry no argtypes, for
    the per-evaluation call: ctypes then passes the caller's ready-made ctypes objects
    without converting each argument (about 1.5 µs less per call). Callers pass exactly
    the C types (c_void_p handle, int, ctypes arrays, byref)."""
    global _raw
    if _raw is None:
        L = load()
        R = ctypes.CDLL(L._name)
        R.mi_metric_value_and_derivative.restype = ctypes.c_int
        _raw = R
    return _raw


def check(status: int, ctx=None):
    if status != MI_OK:
        detail = ""
        if ctx:
            msg = load().mi_last_error(ctx)
            detail = msg.decode() if msg else ""
        raise MiError(status, detail)
