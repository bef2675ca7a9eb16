"""NACA four-digit geometry queries backed by the device.

``NacaFoil`` mirrors the reference class (``core/geometry.py:13-159``): the solver takes
it as ``geometry`` and reads ``.spec``. Masks and signed distances are evaluated by the
library's kernels (the same code the step uses), so host callers see exactly the solid
cells the device steps with.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from foilbench_b200 import _native as N
from foilbench_b200.models import ControlState, FoilSpec


def cell_centers(domain) -> np.ndarray:
    """Cell-centre coordinates (ny, nx, 2) of a domain (reference ``cell_centers``, geometry.py:162)."""
    (x0, x1), (y0, y1) = domain.bounds[0], domain.bounds[1]
    nx, ny = int(domain.resolution[0]), int(domain.resolution[1])
    dx, dy = (x1 - x0) / nx, (y1 - y0) / ny
    xs = np.linspace(x0 + 0.5 * dx, x1 - 0.5 * dx, nx)
    ys = np.linspace(y0 + 0.5 * dy, y1 - 0.5 * dy, ny)
    xx, yy = np.meshgrid(xs, ys)
    return np.stack((xx, yy), axis=-1)


def _grid_desc(domain, spec) -> N.ScenarioDesc:
    d = N.ScenarioDesc()
    d.nx, d.ny = int(domain.resolution[0]), int(domain.resolution[1])
    (d.x0, d.x1), (d.y0, d.y1) = domain.bounds[0], domain.bounds[1]
    axes = tuple(domain.periodic_axes)
    d.periodic_x, d.periodic_y = int("x" in axes), int("y" in axes)
    d.naca = spec.naca.encode("ascii")
    d.chord = float(spec.chord)
    d.pivot_x, d.pivot_y = float(spec.pivot[0]), float(spec.pivot[1])
    d.precision = N.FLOAT64
    d.pressure_scheme = N.PRESSURE_REFERENCE
    d.pressure_tolerance = 1.0e-5
    return d


@dataclass(frozen=True, slots=True)
class NacaFoil:
    spec: FoilSpec

    @property
    def maximum_camber(self) -> float:
        return int(self.spec.naca[0]) / 100.0

    @property
    def camber_position(self) -> float:
        return int(self.spec.naca[1]) / 10.0

    @property
    def thickness(self) -> float:
        return int(self.spec.naca[2:]) / 100.0

    @property
    def maximum_radius(self) -> float:
        """Largest distance from the pivot reached by the section (geometry.py:29-33)."""
        vertical = (self.maximum_camber + 0.51 * self.thickness) * self.spec.chord
        return float(np.hypot(0.75 * self.spec.chord, vertical))

    def signed_distance(self, points: np.ndarray, angle_degrees: float) -> np.ndarray:
        pts = np.ascontiguousarray(np.asarray(points, dtype=np.float64)[:, :2])
        out = np.empty(pts.shape[0], dtype=np.float64)
        ctx = N.default_context()
        N.check(N.lib().fb_naca_signed_distance(ctx.handle, self.spec.naca.encode("ascii"), float(self.spec.chord),
                                                float(self.spec.pivot[0]), float(self.spec.pivot[1]), N.dptr(pts),
                                                pts.shape[0], float(angle_degrees), N.dptr(out)),
                "fb_naca_signed_distance")
        return np.asarray(out, dtype=np.asarray(points).dtype if np.asarray(points).dtype.kind == "f" else np.float64)

    def contains(self, points: np.ndarray, angle_degrees: float) -> np.ndarray:
        return self.signed_distance(points, angle_degrees) <= 0.0

    def normals(self, points: np.ndarray, angle_degrees: float) -> np.ndarray:
        """Central-difference gradient of the signed distance (geometry.py:108-126)."""
        pts = np.asarray(points, dtype=np.float64)
        eps = max(self.spec.chord * 1.0e-4, 1.0e-6)
        ox = np.asarray([eps, 0.0])
        oy = np.asarray([0.0, eps])
        gx = self.signed_distance(pts + ox, angle_degrees) - self.signed_distance(pts - ox, angle_degrees)
        gy = self.signed_distance(pts + oy, angle_degrees) - self.signed_distance(pts - oy, angle_degrees)
        grad = np.stack((gx, gy), axis=1)
        length = np.linalg.norm(grad, axis=1, keepdims=True)
        flat = length[:, 0] < eps
        if np.any(flat):
            a = np.deg2rad(angle_degrees)
            grad[flat, 0] = -np.sin(a)
            grad[flat, 1] = np.cos(a)
            length[flat, 0] = 1.0
        return grad / np.maximum(length, eps)

    def wall_velocity(self, points: np.ndarray, control: ControlState) -> np.ndarray:
        """Rigid rotation about the pivot (geometry.py:131-139)."""
        rel = points[:, :2] - np.asarray(self.spec.pivot[:2], dtype=points.dtype)
        w = np.deg2rad(control.angular_velocity_degrees)
        out = np.empty_like(rel)
        out[:, 0] = -w * rel[:, 1]
        out[:, 1] = w * rel[:, 0]
        return out

    def mask(self, domain, angle_degrees: float) -> np.ndarray:
        """Solid cells (ny, nx) at the cell centres, computed by the device mask kernel."""
        d = _grid_desc(domain, self.spec)
        out = np.empty((d.ny, d.nx), dtype=np.uint8)
        ctx = N.default_context()
        N.check(N.lib().fb_compute_mask(ctx.handle, d, float(angle_degrees), N.u8ptr(out), out.size), "fb_compute_mask")
        return out.astype(bool)
