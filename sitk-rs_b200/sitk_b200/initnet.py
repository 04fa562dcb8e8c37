"""Learned initialiser: a small 3-D convolutional network that proposes the affine a
registration starts from, trained on synthetic pairs the library generates and
registers itself.

The reference starts every registration from CenteredTransformInitializer
(registration/initializer.rs:56-105); this module adds a learned proposal in front of
the same regular-step optimizer, and the acceptance rule keeps the plain optimizer
as the judge: a proposal is used only when its refined result reaches the plain
run's final metric value within a tolerance.

The network (csrc/initnet.cu) reads a fixed/moving pair resampled to 32³ and
normalised (`prepare`), and outputs 12 numbers: the affine matrix minus identity
over MATRIX_SCALE and the translation over TRANSLATION_SCALE (`encode`/`decode`),
in the parameterisation of the centred affine about the fixed image's centre.
Device buffers are torch CUDA tensors; every computation runs in the library.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .metric import DeviceImage, default_context

MATRIX_SCALE = 0.25
TRANSLATION_SCALE = 20.0
GRID = 32
N_LAYERS = 6
# (out, in) of each layer's weight matrix
LAYER_SHAPES = [(16, 27 * 2), (32, 27 * 16), (64, 27 * 32), (128, 27 * 64), (256, 1024), (12, 256)]


def _bind():
    L = _lib.load()
    if getattr(L, "_initnet_bound", False):
        return L
    vp = ctypes.c_void_p
    P = ctypes.POINTER
    fp = P(ctypes.c_float)
    L.mi_initnet_create.argtypes = [vp, ctypes.c_uint64, ctypes.c_int, P(vp)]
    L.mi_initnet_destroy.argtypes = [vp]
    L.mi_initnet_get.argtypes = [vp, ctypes.c_int, ctypes.c_int, fp, fp]
    L.mi_initnet_set.argtypes = [vp, ctypes.c_int, fp, fp]
    L.mi_initnet_forward.argtypes = [vp, ctypes.c_int, vp, vp]
    L.mi_initnet_train_step.argtypes = [vp, ctypes.c_int, vp, vp, ctypes.c_float, fp]
    L.mi_initnet_prepare.argtypes = [vp, vp, vp, vp]
    for f in ("mi_initnet_create", "mi_initnet_destroy", "mi_initnet_get", "mi_initnet_set", "mi_initnet_forward",
              "mi_initnet_train_step", "mi_initnet_prepare"):
        getattr(L, f).restype = ctypes.c_int
    L._initnet_bound = True
    return L


def _check_input(x, batch_dims: int):
    import torch
    if not (isinstance(x, torch.Tensor) and x.is_cuda and x.dtype == torch.float32 and x.is_contiguous()):
        raise ValueError("expected a contiguous float32 CUDA tensor")
    return x


def encode(params: np.ndarray) -> np.ndarray:
    """Affine parameters (…, 12: matrix row-major, translation) → network targets."""
    p = np.asarray(params, dtype=np.float64)
    out = np.empty(p.shape)
    out[..., :9] = (p[..., :9] - np.eye(3).ravel()) / MATRIX_SCALE
    out[..., 9:] = p[..., 9:] / TRANSLATION_SCALE
    return out


def decode(y: np.ndarray) -> np.ndarray:
    """Network outputs (…, 12) → affine parameters."""
    y = np.asarray(y, dtype=np.float64)
    out = np.empty(y.shape)
    out[..., :9] = y[..., :9] * MATRIX_SCALE + np.eye(3).ravel()
    out[..., 9:] = y[..., 9:] * TRANSLATION_SCALE
    return out


def prepare(fixed: DeviceImage, moving: DeviceImage, out=None):
    """The network input of one pair: a (32, 32, 32, 2) float32 CUDA tensor (mi_initnet_prepare)."""
    import torch
    L = _bind()
    if out is None:
        out = torch.empty((GRID, GRID, GRID, 2), dtype=torch.float32, device="cuda")
    _check_input(out, 0)
    torch.cuda.synchronize()
    _lib.check(L.mi_initnet_prepare(fixed.ctx.handle, fixed.handle, moving.handle, out.data_ptr()), fixed.ctx.handle)
    return out


class InitNet:
    """The network and its optimizer state (mi_initnet_*)."""

    def __init__(self, seed: int = 0, max_batch: int = 64, ctx=None):
        L = _bind()
        self.ctx = ctx or default_context()
        self.max_batch = max_batch
        h = ctypes.c_void_p()
        _lib.check(L.mi_initnet_create(self.ctx.handle, int(seed) & (2**64 - 1), int(max_batch), ctypes.byref(h)),
                   self.ctx.handle)
        self.handle = h

    def forward(self, x):
        """x: (B, 32, 32, 32, 2) CUDA float32 → (B, 12) CUDA float32."""
        import torch
        _check_input(x, 1)
        B = x.shape[0]
        out = torch.empty((B, 12), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        _lib.check(_bind().mi_initnet_forward(self.handle, B, x.data_ptr(), out.data_ptr()), self.ctx.handle)
        return out

    def train_step(self, x, target, lr: float) -> float:
        """One forward/backward/Adam step on a batch; returns the batch's mean squared error."""
        import torch
        _check_input(x, 1)
        _check_input(target, 1)
        loss = ctypes.c_float()
        torch.cuda.synchronize()
        _lib.check(_bind().mi_initnet_train_step(self.handle, x.shape[0], x.data_ptr(), target.data_ptr(), float(lr),
                                                 ctypes.byref(loss)), self.ctx.handle)
        return loss.value

    def get(self, which: int, grads: bool = False):
        """(W (out × in), b) of layer `which` as float32 arrays, or their last gradients."""
        o, i = LAYER_SHAPES[which]
        w = np.zeros((o, i), dtype=np.float32)
        b = np.zeros(o, dtype=np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        _lib.check(_bind().mi_initnet_get(self.handle, which, 1 if grads else 0, w.ctypes.data_as(fp),
                                          b.ctypes.data_as(fp)), self.ctx.handle)
        return w, b

    def set(self, which: int, w, b):
        o, i = LAYER_SHAPES[which]
        w = np.ascontiguousarray(w, dtype=np.float32).reshape(o, i)
        b = np.ascontiguousarray(b, dtype=np.float32).reshape(o)
        fp = ctypes.POINTER(ctypes.c_float)
        _lib.check(_bind().mi_initnet_set(self.handle, which, w.ctypes.data_as(fp), b.ctypes.data_as(fp)),
                   self.ctx.handle)

    def state(self):
        return [self.get(l) for l in range(N_LAYERS)]

    def load_state(self, state):
        for l, (w, b) in enumerate(state):
            self.set(l, w, b)

    def propose(self, x) -> np.ndarray:
        """Affine parameters (B × 12) for network inputs x."""
        return decode(self.forward(x).double().cpu().numpy())

    def close(self):
        if getattr(self, "handle", None):
            _bind().mi_initnet_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
