"""Learned initialiser: a small 3-D convolutional network that proposes the affine a
registration starts from, trained on synthetic pairs the library generates and
registers itself.

The reference starts every registration from CenteredTransformInitializer
(registration/initializer.rs:56-105); this module adds a learned proposal in front of
the same regular-step optimizer, and the acceptance rule keeps the plain optimizer
as the arbiter: a proposal is used only when its refined result reaches the plain
run's final metric value within a tolerance.

The network (csrc/initnet.cu) reads a fixed/moving pair resampled to 32³ and
normalised (`prepare`), and outputs 12 numbers: the affine matrix minus identity
over MATRIX_SCALE and the translation over TRANSLATION_SCALE (`encode`/`decode`),
in the parameterisation of the centred affine about the fixed image's centre.
Device buffers are torch CUDA tensors; every computation runs in the library.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass

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

    def save(self, path: str, **meta) -> None:
        """Weights and biases of every layer (float32) into an .npz file, with `meta`
        (strings or numbers describing how they were trained)."""
        arrays = {}
        for l, (w, b) in enumerate(self.state()):
            arrays[f"w{l}"] = w
            arrays[f"b{l}"] = b
        for k, v in meta.items():
            arrays[f"meta_{k}"] = np.asarray(v)
        np.savez_compressed(path, **arrays)

    def load(self, path: str) -> dict:
        """Weights written by save(); returns the stored meta entries."""
        with np.load(path) as z:
            self.load_state([(z[f"w{l}"], z[f"b{l}"]) for l in range(N_LAYERS)])
            return {k[5:]: z[k].item() if z[k].ndim == 0 else z[k].tolist() for k in z.files if k.startswith("meta_")}

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


# ---------------------------------------------------------------------------
# Training data, training and the comparison with the centred initialiser
# ---------------------------------------------------------------------------

@dataclass
class PairSpec:
    """Synthetic pairs: n³ blob phantoms (unit spacing, zero origin) under a random
    centred affine (rotation ±rot_deg about each axis, per-axis scale, translation
    ±trans_mm per axis), counter-based noise; built on the device."""
    n: int = 128
    nblobs: int = 40
    rot_deg: float = 20.0
    trans_mm: float = 20.0
    scale: tuple = (0.9, 1.1)
    noise: float = 5.0


@dataclass
class PlainRun:
    """The plain registration: Mattes metric (bins, random sampling) and regular-step
    gradient descent with physical-shift scales and an estimated learning rate."""
    bins: int = 50
    percentage: float = 0.1
    iterations: int = 200
    minimum_step: float = 1e-4
    gradient_tolerance: float = 1e-4
    relaxation: float = 0.5


def truth_params(matrix, translation) -> np.ndarray:
    """The affine (about the grid centre) that maps fixed points onto moving points for
    a pair whose moving image is base(m·(x − c) + c + t): A = m⁻¹, t' = −m⁻¹·t."""
    mi = np.linalg.inv(np.asarray(matrix, dtype=np.float64))
    return np.concatenate([mi.ravel(), -mi @ np.asarray(translation, dtype=np.float64)])


def identity_params(count: int) -> np.ndarray:
    return np.tile(np.concatenate([np.eye(3).ravel(), np.zeros(3)]), (count, 1))


def target_error(params, truth, center, half: float) -> float:
    """Mean distance (mm) between the two affines' images of the 8 corners of a cube of
    half-width `half` about the centre."""
    p, q = np.asarray(params, dtype=np.float64), np.asarray(truth, dtype=np.float64)
    c = np.asarray(center, dtype=np.float64)
    d = []
    for k in range(8):
        x = c + half * np.array([1 if k & 1 else -1, 1 if k & 2 else -1, 1 if k & 4 else -1], dtype=np.float64)
        y1 = p[:9].reshape(3, 3) @ (x - c) + c + p[9:]
        y2 = q[:9].reshape(3, 3) @ (x - c) + c + q[9:]
        d.append(np.linalg.norm(y1 - y2))
    return float(np.mean(d))


def _pairs(seeds, spec: PairSpec, ctx):
    from . import synth
    fixed, moving, truth = [], [], []
    for s in seeds:
        f, m, p = synth.make_pair_device(spec.n, spec.nblobs, int(s), spec.rot_deg, spec.trans_mm, spec.scale,
                                         spec.noise, ctx=ctx)
        fixed.append(f)
        moving.append(m)
        truth.append(truth_params(p.matrix, p.translation))
    return fixed, moving, np.array(truth)


def _batch(fixed, moving, seeds, spec: PairSpec, run: PlainRun):
    from .metric import SAMPLING_RANDOM
    from .registration import BatchRegistration
    c = [(spec.n - 1) / 2.0] * 3
    return BatchRegistration(fixed, moving, bins=run.bins, kind=0, centers=[c] * len(fixed), strategy=SAMPLING_RANDOM,
                             percentage=run.percentage, seeds=[int(s) for s in seeds])


def _register(br, start, run: PlainRun):
    return br.register(start, iterations=run.iterations, minimum_step=run.minimum_step,
                       gradient_tolerance=run.gradient_tolerance, relaxation=run.relaxation)


def labelled_set(seeds, spec: PairSpec = PairSpec(), run: PlainRun = PlainRun(), ctx=None, batch: int = 64):
    """Network inputs and labels for `seeds`: each pair generated on the device,
    prepared to 32³, and labelled with the plain optimizer's converged parameters
    (run from the generating affine, so the label is the metric's optimum next to the
    truth). Returns dict(x: (N, 32, 32, 32, 2) CUDA tensor, labels, truth (N × 12),
    seconds)."""
    import torch
    ctx = ctx or default_context()
    seeds = list(seeds)
    X = torch.empty((len(seeds), GRID, GRID, GRID, 2), dtype=torch.float32, device="cuda")
    labels = np.empty((len(seeds), 12))
    truths = np.empty((len(seeds), 12))
    t0 = time.perf_counter()
    for a in range(0, len(seeds), batch):
        chunk = seeds[a:a + batch]
        fixed, moving, truth = _pairs(chunk, spec, ctx)
        for i, (f, m) in enumerate(zip(fixed, moving)):
            prepare(f, m, X[a + i])
        br = _batch(fixed, moving, chunk, spec, run)
        p, _ = _register(br, truth, run)
        br.close()
        for img in fixed + moving:
            img.free()
        labels[a:a + len(chunk)] = p
        truths[a:a + len(chunk)] = truth
    torch.cuda.synchronize()
    return {"x": X, "labels": labels, "truth": truths, "seconds": time.perf_counter() - t0}


def train(net: InitNet, X, labels, epochs: int = 20, batch: int = 64, lr: float = 1e-3, lr_final: float = 2e-5,
          seed: int = 0):
    """Mini-batch Adam on the mean squared error of the encoded labels, learning rate
    decayed from lr to lr_final (cosine) over the run. Returns the mean loss of each
    epoch and the seconds spent."""
    import math as _m

    import torch
    n = X.shape[0]
    T = torch.from_numpy(encode(labels).astype(np.float32)).cuda()
    rng = np.random.Generator(np.random.PCG64(seed))
    steps = epochs * (n // batch)
    k = 0
    losses = []
    t0 = time.perf_counter()
    for _ in range(epochs):
        perm = torch.from_numpy(rng.permutation(n)).cuda()
        acc = 0.0
        for a in range(0, n - batch + 1, batch):
            idx = perm[a:a + batch]
            rate = lr_final + 0.5 * (lr - lr_final) * (1.0 + _m.cos(_m.pi * k / max(steps, 1)))
            acc += net.train_step(X[idx].contiguous(), T[idx].contiguous(), rate)
            k += 1
        losses.append(acc / max(n // batch, 1))
    torch.cuda.synchronize()
    return losses, time.perf_counter() - t0


def evaluate(net: InitNet, seeds, spec: PairSpec = PairSpec(), run: PlainRun = PlainRun(), ctx=None,
             batch: int = 64, tolerance: float = 1e-3, single_pairs: int = 8):
    """The learned proposal against the centred initialiser on held-out pairs.

    Per chunk of `batch` pairs (one batched registration object, so both starts see
    the same metric and sampling): the plain run from the centred initialiser (the
    identity about the centre: the images share their geometry), then the network's
    proposal (prepare + forward, timed) refined by the same optimizer. A proposal is
    accepted when its refined metric value is within `tolerance` of the plain run's
    final value or lower (the value is −MI). The first `single_pairs` pairs also run
    through the single-pair driver from both starts with every evaluation recorded:
    the plain GPU form's registrations/s and the iterations each start needs to reach
    the plain run's final value within `tolerance`."""
    import torch

    from . import registration
    from .metric import SAMPLING_RANDOM, DeviceMattesMetric
    from .transforms import AffineTransform
    ctx = ctx or default_context()
    seeds = list(seeds)
    c = [(spec.n - 1) / 2.0] * 3
    half = 0.3 * spec.n
    X = torch.empty((batch, GRID, GRID, GRID, 2), dtype=torch.float32, device="cuda")
    rec = {k: [] for k in ("v_plain", "v_learned", "it_plain", "it_learned", "tre_plain", "tre_learned",
                           "tre_proposal")}
    wall_plain = wall_learned = wall_infer = 0.0
    single = {"plain_s": [], "reach_plain": [], "reach_learned": [], "learned_s": []}
    warm = False
    for a in range(0, len(seeds), batch):
        chunk = seeds[a:a + batch]
        fixed, moving, truth = _pairs(chunk, spec, ctx)
        br = _batch(fixed, moving, chunk, spec, run)
        if not warm:  # autotune and graph capture, untimed
            _register(br, identity_params(len(chunk)), run)
            warm = True
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pp, rp = _register(br, identity_params(len(chunk)), run)
        wall_plain += time.perf_counter() - t0
        t0 = time.perf_counter()
        for i, (f, m) in enumerate(zip(fixed, moving)):
            prepare(f, m, X[i])
        prop = net.propose(X[:len(chunk)])
        wall_infer += time.perf_counter() - t0
        t0 = time.perf_counter()
        pl, rl = _register(br, prop, run)
        wall_learned += time.perf_counter() - t0
        br.close()
        for i in range(len(chunk)):
            rec["v_plain"].append(rp[i].value)
            rec["v_learned"].append(rl[i].value)
            rec["it_plain"].append(rp[i].iterations)
            rec["it_learned"].append(rl[i].iterations)
            rec["tre_plain"].append(target_error(pp[i], truth[i], c, half))
            rec["tre_learned"].append(target_error(pl[i], truth[i], c, half))
            rec["tre_proposal"].append(target_error(prop[i], truth[i], c, half))
        # single-pair driver, every evaluation recorded
        for i in range(min(len(chunk), single_pairs - len(single["plain_s"]))):
            traces = []
            for start, key in ((identity_params(1)[0], "plain_s"), (prop[i], "learned_s")):
                metric = DeviceMattesMetric.from_device_sampled(fixed[i], moving[i], bins=run.bins,
                                                                strategy=SAMPLING_RANDOM, percentage=run.percentage,
                                                                seed=int(chunk[i]))
                t = AffineTransform(start[:9].reshape(3, 3), start[9:], c)
                torch.cuda.synchronize()
                t1 = time.perf_counter()
                r = registration.register_rsgd(metric, t, iterations=run.iterations, minimum_step=run.minimum_step,
                                               gradient_tolerance=run.gradient_tolerance,
                                               relaxation=run.relaxation, record=True)
                single[key].append(time.perf_counter() - t1)
                traces.append((r.value, r.trace[:, 0]))
                metric.close()
            goal = traces[0][0] + tolerance
            for (v, tr), key in zip(traces, ("reach_plain", "reach_learned")):
                hit = np.nonzero(tr <= goal)[0]
                single[key].append(int(hit[0]) + 1 if hit.size else None)
        for img in fixed + moving:
            img.free()
    v_p, v_l = np.array(rec["v_plain"]), np.array(rec["v_learned"])
    accepted = v_l <= v_p + tolerance
    n = len(seeds)
    reached = [r for r in single["reach_learned"] if r is not None]

    def stats(v):
        v = np.asarray(v, dtype=np.float64)
        return {"mean": float(v.mean()), "p50": float(np.median(v)), "p90": float(np.percentile(v, 90))}

    return {
        "pairs": n,
        "accepted": float(accepted.mean()),
        "learned_better_by_1e-3": float((v_l < v_p - tolerance).mean()),
        "iterations": {"plain": stats(rec["it_plain"]), "learned": stats(rec["it_learned"])},
        "tre_mm": {"plain": stats(rec["tre_plain"]), "proposal": stats(rec["tre_proposal"]),
                   "learned": stats(rec["tre_learned"])},
        "within_1mm": {"plain": float(np.mean(np.array(rec["tre_plain"]) < 1.0)),
                       "learned": float(np.mean(np.array(rec["tre_learned"]) < 1.0))},
        "batched_s": {"plain": wall_plain, "learned_refine": wall_learned, "inference": wall_infer},
        "registrations_per_s": {
            "batched_plain": n / wall_plain,
            "batched_learned": n / (wall_learned + wall_infer),
            "single_pair_plain": len(single["plain_s"]) / max(sum(single["plain_s"]), 1e-12),
            "single_pair_learned": len(single["learned_s"]) / max(sum(single["learned_s"]), 1e-12),
        },
        "single_pair_iterations_to_plain_final": {
            "pairs": len(single["plain_s"]),
            "plain": float(np.mean(single["reach_plain"])) if single["reach_plain"] else None,
            "learned": float(np.mean(reached)) if reached else None,
            "learned_reached": len(reached),
        },
        "values": {"plain_mean": float(v_p.mean()), "learned_mean": float(v_l.mean())},
    }
