"""Seeded synthetic registration pairs (blob phantoms under a random affine).

No public dataset is involved in this metric's benchmarks: the workloads are blob
phantoms — a linear ramp background plus Gaussian blobs (σ 3–10 voxels, amplitude
U[50, 200]) plus N(0, 5) noise — and a moving image that is the fixed image
resampled (trilinear, clamp-to-edge) through a random centred affine, with
independent noise. Everything derives from one numpy PCG64 stream per pair, drawn in
a fixed order (blob parameters, fixed noise, affine, moving noise), so a pair is
bit-reproducible from its seed.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

MASTER_SEED = 20261203


@dataclass
class Pair:
    fixed: np.ndarray      # float32 [z, y, x]
    moving: np.ndarray     # float32 [z, y, x]
    matrix: np.ndarray     # 3×3 of the generating affine (moving(x) = fixed(A(x−c)+c+t))
    translation: np.ndarray
    center: np.ndarray
    spacing: tuple = (1.0, 1.0, 1.0)
    origin: tuple = (0.0, 0.0, 0.0)


def blob_params(n: int, nblobs: int, rng: np.random.Generator) -> np.ndarray:
    """Per blob (σ, amplitude, cx, cy, cz), drawn in that order from `rng`."""
    out = np.empty((nblobs, 5))
    for b in range(nblobs):
        out[b, 0] = rng.uniform(3.0, 10.0)
        out[b, 1] = rng.uniform(50.0, 200.0)
        out[b, 2:5] = rng.uniform(0.0, n - 1, size=3)  # (x, y, z)
    return out


def render_phantom(n: int, blobs: np.ndarray) -> np.ndarray:
    """Ramp background plus the given Gaussian blobs on an n³ grid (float64); each blob
    is added inside its ±3.5σ box, blobs in order."""
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    vol = 20.0 + 40.0 * (x + 0.5 * y + 0.25 * z) / (1.75 * max(n - 1, 1))
    del x, y, z
    for sigma, amp, cx, cy, cz in blobs:
        c = (cx, cy, cz)
        r = int(math.ceil(3.5 * sigma))
        lo = [max(int(c[d]) - r, 0) for d in range(3)]
        hi = [min(int(c[d]) + r + 1, n) for d in range(3)]
        xs = np.arange(lo[0], hi[0]) - c[0]
        ys = np.arange(lo[1], hi[1]) - c[1]
        zs = np.arange(lo[2], hi[2]) - c[2]
        g = np.exp(-0.5 * (zs[:, None, None] ** 2 + ys[None, :, None] ** 2 + xs[None, None, :] ** 2) / sigma ** 2)
        vol[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] += amp * g
    return vol


def blob_phantom(n: int, nblobs: int, rng: np.random.Generator) -> np.ndarray:
    """Ramp background plus `nblobs` Gaussian blobs on an n³ grid (float64)."""
    return render_phantom(n, blob_params(n, nblobs, rng))


def rotation_xyz(ax: float, ay: float, az: float) -> np.ndarray:
    cx, sx, cy, sy, cz, sz = math.cos(ax), math.sin(ax), math.cos(ay), math.sin(ay), math.cos(az), math.sin(az)
    rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return rz @ rx @ ry


def random_affine(rng: np.random.Generator, rot_deg: float, scale: tuple | None, trans_mm: float):
    ang = np.deg2rad(rng.uniform(-rot_deg, rot_deg, size=3))
    m = rotation_xyz(*ang)
    if scale is not None:
        m = m @ np.diag(rng.uniform(scale[0], scale[1], size=3))
    t = rng.uniform(-trans_mm, trans_mm, size=3)
    return m, t


def resample_linear(vol: np.ndarray, m: np.ndarray, t: np.ndarray, center: np.ndarray) -> np.ndarray:
    """out(x) = vol(m·(x − center) + center + t), trilinear, clamp-to-edge, unit
    spacing and zero origin (index = physical). Processed slab by slab."""
    nz, ny, nx = vol.shape
    out = np.empty(vol.shape, dtype=np.float64)
    ys, xs = np.meshgrid(np.arange(ny, dtype=np.float64), np.arange(nx, dtype=np.float64), indexing="ij")
    for z0 in range(0, nz, 16):
        z1 = min(z0 + 16, nz)
        zz = np.arange(z0, z1, dtype=np.float64)[:, None, None]
        px = xs[None] - center[0]
        py = ys[None] - center[1]
        pz = zz - center[2]
        q = [m[r, 0] * px + m[r, 1] * py + m[r, 2] * pz + center[r] + t[r] for r in range(3)]
        qx, qy, qz = [np.broadcast_to(a, (z1 - z0, ny, nx)) for a in q]
        qx = np.clip(qx, 0.0, nx - 1.0)
        qy = np.clip(qy, 0.0, ny - 1.0)
        qz = np.clip(qz, 0.0, nz - 1.0)
        x0 = np.minimum(np.floor(qx).astype(np.int64), nx - 2)
        y0 = np.minimum(np.floor(qy).astype(np.int64), ny - 2)
        z0i = np.minimum(np.floor(qz).astype(np.int64), nz - 2)
        fx, fy, fz = qx - x0, qy - y0, qz - z0i
        acc = np.zeros((z1 - z0, ny, nx))
        for dz in (0, 1):
            wz = fz if dz else 1.0 - fz
            for dy in (0, 1):
                wy = fy if dy else 1.0 - fy
                for dx in (0, 1):
                    wx = fx if dx else 1.0 - fx
                    acc += wz * wy * wx * vol[z0i + dz, y0 + dy, x0 + dx]
        out[z0:z1] = acc
    return out


def make_pair(n: int, nblobs: int, seed: int, rot_deg: float, trans_mm: float,
              scale: tuple | None = (0.95, 1.05), noise: float = 5.0) -> Pair:
    rng = np.random.Generator(np.random.PCG64(seed))
    base = blob_phantom(n, nblobs, rng)
    fixed = base + rng.normal(0.0, noise, size=base.shape)
    m, t = random_affine(rng, rot_deg, scale, trans_mm)
    center = np.full(3, (n - 1) / 2.0)
    moving = resample_linear(base, m, t, center) + rng.normal(0.0, noise, size=base.shape)
    return Pair(fixed.astype(np.float32), moving.astype(np.float32), m, t, center)


def config0_pair(seed: int = MASTER_SEED) -> Pair:
    """64³, 20 blobs, rotation ±10°, scale 0.95–1.05, translation ±5 mm."""
    return make_pair(64, 20, seed, 10.0, 5.0, (0.95, 1.05))


def config1_pair(seed: int = MASTER_SEED, n: int = 256) -> Pair:
    """256³, 60 blobs, rigid: rotation ±15°, translation ±12 mm."""
    return make_pair(n, 60, seed, 15.0, 12.0, None)


# ---------------------------------------------------------------------------
# Counter-based variant, with a device twin (mi_synth_pair): the blob parameters and
# the affine come from the pair's PCG64 stream as above (blobs first, then the
# affine), but the noise of voxel i is a pure function of (seed, field, i) — a
# SplitMix64-mixed counter turned into a normal by Box–Muller — so a GPU can produce
# the same volumes without replaying a sequential stream. The two agree to the
# rounding of exp/log/cos.
# ---------------------------------------------------------------------------
_GAMMA = np.uint64(0x9E3779B97F4A7C15)


def _mix64(z: np.ndarray) -> np.ndarray:
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def noise_key(seed: int, field: int) -> int:
    """The counter key of a noise field (1 = fixed, 2 = moving) of a pair."""
    with np.errstate(over="ignore"):
        return int(_mix64(np.array([seed], dtype=np.uint64) + np.uint64(field) * _GAMMA)[0])


def counter_normal(key: int, count: int) -> np.ndarray:
    """N(0, 1) draws i = 0..count−1: u1, u2 from the mixed counters key + (2i+1)·γ and
    key + (2i+2)·γ (53-bit fractions), z = sqrt(−2 ln(1 − u1))·cos(2π u2)."""
    i = np.arange(count, dtype=np.uint64)
    k = np.uint64(key)
    with np.errstate(over="ignore"):
        a = _mix64(k + (np.uint64(2) * i + np.uint64(1)) * _GAMMA)
        b = _mix64(k + (np.uint64(2) * i + np.uint64(2)) * _GAMMA)
    u1 = (a >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    u2 = (b >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    return np.sqrt(-2.0 * np.log(1.0 - u1)) * np.cos(2.0 * math.pi * u2)


def counter_pair_params(n: int, nblobs: int, seed: int, rot_deg: float, trans_mm: float,
                        scale: tuple | None = (0.95, 1.05)):
    """(blobs, matrix, translation, centre) of a counter-based pair."""
    rng = np.random.Generator(np.random.PCG64(seed))
    blobs = blob_params(n, nblobs, rng)
    m, t = random_affine(rng, rot_deg, scale, trans_mm)
    return blobs, m, t, np.full(3, (n - 1) / 2.0)


def make_pair_counter(n: int, nblobs: int, seed: int, rot_deg: float, trans_mm: float,
                      scale: tuple | None = (0.95, 1.05), noise: float = 5.0) -> Pair:
    """CPU reference of the counter-based pair (the device builds the same pair with
    make_pair_device)."""
    blobs, m, t, center = counter_pair_params(n, nblobs, seed, rot_deg, trans_mm, scale)
    base = render_phantom(n, blobs)
    fixed = base + noise * counter_normal(noise_key(seed, 1), n ** 3).reshape(base.shape)
    moving = resample_linear(base, m, t, center) + noise * counter_normal(noise_key(seed, 2), n ** 3).reshape(base.shape)
    return Pair(fixed.astype(np.float32), moving.astype(np.float32), m, t, center)


def make_pair_device(n: int, nblobs: int, seed: int, rot_deg: float, trans_mm: float,
                     scale: tuple | None = (0.95, 1.05), noise: float = 5.0, ctx=None):
    """The counter-based pair built on the device (mi_synth_pair): returns
    (fixed DeviceImage, moving DeviceImage, Pair with the truth and no volumes)."""
    import ctypes
    from . import _lib
    from .metric import DeviceImage, default_context
    ctx = ctx or default_context()
    blobs, m, t, center = counter_pair_params(n, nblobs, seed, rot_deg, trans_mm, scale)
    L = _lib.load()
    if not getattr(L, "_synth_bound", False):
        P = ctypes.POINTER
        L.mi_synth_pair.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, P(ctypes.c_double),
                                    P(ctypes.c_double), ctypes.c_uint64, ctypes.c_double, P(ctypes.c_void_p),
                                    P(ctypes.c_void_p)]
        L.mi_synth_pair.restype = ctypes.c_int
        L._synth_bound = True
    b = np.ascontiguousarray(blobs, dtype=np.float64)
    a = np.ascontiguousarray(np.concatenate([np.asarray(m, dtype=np.float64).ravel(), np.asarray(t, dtype=np.float64)]))
    hf, hm = ctypes.c_void_p(), ctypes.c_void_p()
    dp = ctypes.POINTER(ctypes.c_double)
    _lib.check(L.mi_synth_pair(ctx.handle, n, len(b), b.ctypes.data_as(dp), a.ctypes.data_as(dp),
                               int(seed) & (2**64 - 1), float(noise), ctypes.byref(hf), ctypes.byref(hm)), ctx.handle)
    geo_f, geo_m = _lib.MiGeometry(), _lib.MiGeometry()
    _lib.check(L.mi_image_geometry(hf, ctypes.byref(geo_f)))
    _lib.check(L.mi_image_geometry(hm, ctypes.byref(geo_m)))
    return DeviceImage(hf, ctx, geo_f), DeviceImage(hm, ctx, geo_m), Pair(None, None, m, t, center)
