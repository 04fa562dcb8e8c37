"""Transform families the device metric differentiates (transform/parametric.rs).

Each class holds what the reference type holds — the parameter vector and the fixed
parameters — with the reference's parameter order, and hands the library its kind
code. The matrix, offset and Jacobian are formed by the library (csrc/transforms.cpp),
in the reference's operation order.
"""
from __future__ import annotations

import math

import numpy as np

AFFINE, EULER3D, VERSOR_RIGID3D, TRANSLATION = 0, 1, 2, 3


class ParametricTransform:
    kind: int = -1
    nparams: int = 0

    def __init__(self, params, fixed_params):
        self.params = np.asarray(params, dtype=np.float64).copy()
        self.fixed_params = np.asarray(fixed_params, dtype=np.float64).copy()
        if self.params.size != self.nparams:
            raise ValueError(f"{type(self).__name__} takes {self.nparams} parameters")

    def number_of_parameters(self) -> int:
        return self.nparams

    def parameters(self) -> np.ndarray:
        return self.params.copy()

    def set_parameters(self, p) -> None:
        p = np.asarray(p, dtype=np.float64)
        if p.size != self.nparams:
            raise ValueError("parameter count mismatch")  # TransformError::InvalidParameters
        self.params = p.copy()

    def set_fixed_parameters(self, fp) -> None:
        self.fixed_params = np.asarray(fp, dtype=np.float64).copy()

    def center(self) -> np.ndarray:
        return self.fixed_params[:3].copy()


class AffineTransform(ParametricTransform):
    """y = A·(x − c) + t + c; params = A row-major (9), t (3); fixed = c
    (parametric.rs:473-608)."""
    kind = AFFINE
    nparams = 12

    def __init__(self, matrix=None, translation=(0.0, 0.0, 0.0), center=(0.0, 0.0, 0.0)):
        m = np.eye(3) if matrix is None else np.asarray(matrix, dtype=np.float64).reshape(3, 3)
        super().__init__(np.concatenate([m.ravel(), np.asarray(translation, dtype=np.float64)]), center)


class Euler3DTransform(ParametricTransform):
    """Rotation Rz·Rx·Ry about c, then t; params = (ax, ay, az, tx, ty, tz);
    fixed = c (+ computeZYX) (parametric.rs:935-1180)."""
    kind = EULER3D
    nparams = 6

    def __init__(self, angles=(0.0, 0.0, 0.0), translation=(0.0, 0.0, 0.0), center=(0.0, 0.0, 0.0),
                 compute_zyx: bool = False):
        fp = list(center) + ([1.0] if compute_zyx else [])
        super().__init__(list(angles) + list(translation), fp)


class VersorRigid3DTransform(ParametricTransform):
    """Versor rotation about c, then t; params = (vx, vy, vz, tx, ty, tz);
    fixed = c (parametric.rs:1211-1437)."""
    kind = VERSOR_RIGID3D
    nparams = 6

    def __init__(self, versor=(0.0, 0.0, 0.0), translation=(0.0, 0.0, 0.0), center=(0.0, 0.0, 0.0)):
        super().__init__(list(versor) + list(translation), center)

    @staticmethod
    def versor_from_axis_angle(axis, angle):
        a = np.asarray(axis, dtype=np.float64)
        a = a / np.linalg.norm(a)
        return a * math.sin(angle / 2.0)


class TranslationTransform(ParametricTransform):
    kind = TRANSLATION
    nparams = 3

    def __init__(self, translation=(0.0, 0.0, 0.0)):
        super().__init__(translation, [])


class BSplineTransform:
    """Cubic B-spline free-form deformation (transform/bspline.rs): a control-point grid
    (size = mesh + 3 per axis) with one coefficient per control point and dimension;
    x ↦ x + Σ_k w_k(x)·c_k over the 4³ control points whose support covers x, identity
    outside the grid's valid region. Parameters are the coefficients, dimension-major
    ([all x][all y][all z], each grid x-fastest); fixed parameters are the grid's
    [size(3), origin(3), spacing(3), direction(9)], as ITK lays them out."""

    BSPLINE = 4  # no affine form: evaluated through its own device path

    def __init__(self, domain_origin, domain_physical_dimensions, domain_direction, mesh_size):
        """BSplineTransform::new (bspline.rs:229-272)."""
        mesh = [int(m) for m in mesh_size]
        if len(mesh) != 3 or min(mesh) < 1:
            raise ValueError("InvalidBSplineDomain: three positive mesh sizes")
        d = [float(v) for v in np.asarray(domain_direction, dtype=np.float64).ravel()]
        size = [m + 3 for m in mesh]
        spacing = [float(domain_physical_dimensions[i]) / float(mesh[i]) for i in range(3)]
        shift = [-0.5 * spacing[i] * (3.0 - 1.0) for i in range(3)]
        rotated = []
        for r in range(3):  # core/matrix.rs mat_vec: from 0.0, columns in order
            acc = 0.0
            for c in range(3):
                acc += d[r * 3 + c] * shift[c]
            rotated.append(acc)
        origin = [float(domain_origin[i]) + rotated[i] for i in range(3)]
        self.fixed_params = np.array([float(v) for v in size] + origin + spacing + d, dtype=np.float64)
        self.grid_size = tuple(size)
        self.params = np.zeros(3 * size[0] * size[1] * size[2])
        self.nparams = self.params.size

    @classmethod
    def from_image_domain(cls, geo, mesh_size):
        """BSplineTransform::from_image_domain (bspline.rs:324-336): the domain is the
        image's origin, direction and size·spacing."""
        phys = [float(geo.size[i]) * float(geo.spacing[i]) for i in range(3)]
        return cls([geo.origin[i] for i in range(3)], phys, [geo.direction[i] for i in range(9)], mesh_size)

    def number_of_parameters(self) -> int:
        return self.nparams

    def parameters(self) -> np.ndarray:
        return self.params.copy()

    def set_parameters(self, p) -> None:
        p = np.asarray(p, dtype=np.float64)
        if p.size != self.nparams:
            raise ValueError("parameter count mismatch")
        self.params = p.ravel().copy()
