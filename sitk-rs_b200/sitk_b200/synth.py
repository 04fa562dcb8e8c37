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


def blob_phantom(n: int, nblobs: int, rng: np.random.Generator) -> np.ndarray:
    """Ramp background plus `nblobs` Gaussian blobs on an n³ grid (float64)."""
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    vol = 20.0 + 40.0 * (x + 0.5 * y + 0.25 * z) / (1.75 * max(n - 1, 1))
    del x, y, z
    for _ in range(nblobs):
        sigma = rng.uniform(3.0, 10.0)
        amp = rng.uniform(50.0, 200.0)
        c = rng.uniform(0.0, n - 1, size=3)  # (x, y, z)
        r = int(math.ceil(3.5 * sigma))
        lo = [max(int(c[d]) - r, 0) for d in range(3)]
        hi = [min(int(c[d]) + r + 1, n) for d in range(3)]
        xs = np.arange(lo[0], hi[0]) - c[0]
        ys = np.arange(lo[1], hi[1]) - c[1]
        zs = np.arange(lo[2], hi[2]) - c[2]
        g = np.exp(-0.5 * (zs[:, None, None] ** 2 + ys[None, :, None] ** 2 + xs[None, None, :] ** 2) / sigma ** 2)
        vol[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] += amp * g
    return vol


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
