"""B200-native Mattes mutual-information metric for sitk-rs registration.

The compute path is libmi_b200.so (CUDA, sm_100a) behind the C ABI in
include/mi_b200.h; this package is the host-side mirror of the reference's device
metric seam (crates/sitk/src/registration/device.rs) over that ABI.
"""
from .metric import (Context, DeviceImage, DeviceMattesMetric, DeviceMeanSquaresMetric, DeviceCorrelationMetric,
                     MetricValue, default_context,
                     geometry, transform_stage, transform_form, SAMPLING_NONE, SAMPLING_REGULAR, SAMPLING_RANDOM,
                     SAMPLING_EXPLICIT)
from .transforms import (AffineTransform, Euler3DTransform, ParametricTransform,
                         TranslationTransform, VersorRigid3DTransform)
from ._lib import MiError

__all__ = [
    "Context", "DeviceImage", "DeviceMattesMetric", "DeviceMeanSquaresMetric", "DeviceCorrelationMetric",
    "MetricValue", "default_context", "geometry",
    "transform_stage", "transform_form", "AffineTransform", "Euler3DTransform", "ParametricTransform",
    "TranslationTransform", "VersorRigid3DTransform", "MiError", "SAMPLING_NONE",
    "SAMPLING_REGULAR", "SAMPLING_RANDOM", "SAMPLING_EXPLICIT",
]
