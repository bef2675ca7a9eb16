"""Numpy restatement of the reference Stable Fluids step (CPU oracle).

TEST INFRASTRUCTURE ONLY -- never imported by the product package.

Every function names the reference symbol it restates. Paths are relative to the
reference project root; ``PY/`` abbreviates ``implementations/python/src/foilbench_py/``.
Arithmetic follows the reference's numpy expressions (same dtypes, same operation
order where it matters) so that fixture comparisons can be tight.

Third-party algorithms restated here (not imported):
* ``scipy.sparse.linalg.cg`` (scipy 1.18.0, pinned in
  ``implementations/python/uv.lock``): the textbook preconditioned CG loop, stop
  test ``||r|| < max(atol, rtol*||b||)`` at the top of each iteration, callback
  after each update, ``info = maxiter`` when the loop is exhausted.
* ``scipy.fft.dstn/idstn(type=1, norm="ortho")``: the orthonormal DST-I
  ``X_k = sqrt(2/(n+1)) sum_j x_j sin(pi (j+1)(k+1)/(n+1))`` applied along each
  axis; computed here through the FFT of the odd extension of length 2(n+1).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


class OracleFailure(RuntimeError):
    """Classified numerical failure, restating ``NumericalFailure`` (PY/core/models.py:294-311)."""

    def __init__(self, reason: str, detail: str, stage: str = "postcondition", evidence=None):
        super().__init__(detail)
        self.reason = reason
        self.stage = stage
        self.evidence = {} if evidence is None else dict(evidence)


@dataclass(frozen=True)
class Grid:
    """Uniform 2D MAC grid; restates ``DomainSpec`` (PY/core/models.py:50-93)."""

    nx: int
    ny: int
    x0: float
    x1: float
    y0: float
    y1: float
    periodic_x: bool = False
    periodic_y: bool = False

    @property
    def dx(self) -> float:
        return (self.x1 - self.x0) / self.nx

    @property
    def dy(self) -> float:
        return (self.y1 - self.y0) / self.ny

    @property
    def periodic_axes(self) -> tuple[str, ...]:
        return tuple(a for a, on in (("x", self.periodic_x), ("y", self.periodic_y)) if on)

    @classmethod
    def from_domain(cls, domain) -> "Grid":
        (x0, x1), (y0, y1) = domain.bounds[0], domain.bounds[1]
        nx, ny = int(domain.resolution[0]), int(domain.resolution[1])
        axes = tuple(domain.periodic_axes)
        return cls(nx, ny, float(x0), float(x1), float(y0), float(y1), "x" in axes, "y" in axes)


# --------------------------------------------------------------------------- geometry


def cell_centers(grid: Grid) -> np.ndarray:
    """Cell-centre coordinates (ny, nx, 2); ``cell_centers`` PY/core/geometry.py:162-168."""
    xs = np.linspace(grid.x0 + 0.5 * grid.dx, grid.x1 - 0.5 * grid.dx, grid.nx)
    ys = np.linspace(grid.y0 + 0.5 * grid.dy, grid.y1 - 0.5 * grid.dy, grid.ny)
    xx, yy = np.meshgrid(xs, ys)
    return np.stack((xx, yy), axis=-1)


def _naca_digits(naca: str) -> tuple[float, float, float]:
    """Camber, camber position, thickness; ``NacaFoil`` properties PY/core/geometry.py:16-27."""
    return int(naca[0]) / 100.0, int(naca[1]) / 10.0, int(naca[2:]) / 100.0


def naca_maximum_radius(naca: str, chord: float) -> float:
    """``NacaFoil.maximum_radius`` PY/core/geometry.py:29-33."""
    m, _, t = _naca_digits(naca)
    return float(np.hypot(0.75 * chord, (m + 0.51 * t) * chord))


def naca_surfaces(naca: str, chord: float, x_local: np.ndarray):
    """Upper and lower surface heights; ``NacaFoil.surfaces`` PY/core/geometry.py:60-90."""
    m, p, t = _naca_digits(naca)
    xc = np.clip(x_local / chord, 0.0, 1.0)
    half = 5.0 * t * chord * (
        0.2969 * np.sqrt(np.maximum(xc, 0.0))
        - 0.1260 * xc
        - 0.3516 * xc**2
        + 0.2843 * xc**3
        - 0.1036 * xc**4
    )
    camber = np.zeros_like(xc)
    if m > 0.0 and p > 0.0:
        front = xc < p
        xf, xb = xc[front], xc[~front]
        camber[front] = m / p**2 * (2.0 * p * xf - xf**2)
        camber[~front] = m / (1.0 - p) ** 2 * ((1.0 - 2.0 * p) + 2.0 * p * xb - xb**2)
        camber *= chord
    return camber + half, camber - half


def _to_local(points: np.ndarray, pivot, chord: float, angle_degrees: float) -> np.ndarray:
    """Pivot-relative rotation into the chord frame; ``NacaFoil._to_local`` PY/core/geometry.py:35-44."""
    angle = np.deg2rad(angle_degrees)
    c, s = np.cos(angle), np.sin(angle)
    rel = points[:, :2] - np.asarray(pivot[:2], dtype=points.dtype)
    out = np.empty_like(rel)
    out[:, 0] = c * rel[:, 0] + s * rel[:, 1]
    out[:, 1] = -s * rel[:, 0] + c * rel[:, 1]
    out[:, 0] += 0.25 * chord
    return out


def naca_signed_distance(naca: str, chord: float, pivot, points: np.ndarray, angle_degrees: float):
    """Approximate signed distance; ``NacaFoil.signed_distance`` PY/core/geometry.py:92-106."""
    local = _to_local(points, pivot, chord, angle_degrees)
    upper, lower = naca_surfaces(naca, chord, local[:, 0])
    x, y = local[:, 0], local[:, 1]
    within_chord = (x >= 0.0) & (x <= chord)
    outside_v = np.maximum(y - upper, lower - y)
    inside_v = -np.minimum(upper - y, y - lower)
    vertical = np.where((y <= upper) & (y >= lower), inside_v, outside_v)
    beyond = np.maximum(np.maximum(-x, x - chord), 0.0)
    dist = np.where(within_chord, vertical, np.hypot(beyond, np.maximum(vertical, 0.0)))
    return np.asarray(dist, dtype=points.dtype)


def naca_mask(naca: str, chord: float, pivot, grid: Grid, angle_degrees: float) -> np.ndarray:
    """Solid cells ``sdf <= 0`` at cell centres; ``NacaFoil.mask`` PY/core/geometry.py:157-159."""
    pts = cell_centers(grid).reshape(-1, 2)
    return (naca_signed_distance(naca, chord, pivot, pts, angle_degrees) <= 0.0).reshape(grid.ny, grid.nx)


def wall_velocity_grid(pivot, omega_degrees: float, grid: Grid) -> np.ndarray:
    """Rigid rotation about the pivot at cell centres; ``NacaFoil.wall_velocity`` PY/core/geometry.py:131-139."""
    pts = cell_centers(grid).reshape(-1, 2)
    rel = pts - np.asarray(pivot[:2], dtype=pts.dtype)
    w = np.deg2rad(omega_degrees)
    out = np.empty_like(rel)
    out[:, 0] = -w * rel[:, 1]
    out[:, 1] = w * rel[:, 0]
    return out.reshape(grid.ny, grid.nx, 2)


# --------------------------------------------------------------------------- MAC grid


def faces_to_cell(u: np.ndarray, v: np.ndarray) -> np.ndarray:
    """Face averages to cell velocity; ``faces_to_cell`` PY/core/grid.py:25-29."""
    return np.stack((0.5 * (u[:, :-1] + u[:, 1:]), 0.5 * (v[:-1, :] + v[1:, :])), axis=-1)


def cell_to_faces(vel: np.ndarray):
    """Cell velocity to faces, boundary faces copy the adjacent cell; PY/core/grid.py:32-44."""
    ny, nx, _ = vel.shape
    u = np.empty((ny, nx + 1), dtype=vel.dtype)
    v = np.empty((ny + 1, nx), dtype=vel.dtype)
    u[:, 1:-1] = 0.5 * (vel[:, :-1, 0] + vel[:, 1:, 0])
    u[:, 0], u[:, -1] = vel[:, 0, 0], vel[:, -1, 0]
    v[1:-1, :] = 0.5 * (vel[:-1, :, 1] + vel[1:, :, 1])
    v[0, :], v[-1, :] = vel[0, :, 1], vel[-1, :, 1]
    return u, v


def apply_domain_boundaries(u, v, grid: Grid, freestream, channel_walls: bool = False) -> None:
    """Inlet/outlet/far-field/channel/periodic faces in place; PY/core/grid.py:47-78."""
    ux, uy = freestream[0], freestream[1]
    if grid.periodic_x:
        avg = 0.5 * (u[:, 0] + u[:, -1])
        u[:, 0] = avg
        u[:, -1] = avg
    else:
        u[:, 0] = ux
        u[:, -1] = u[:, -2]
        v[:, 0] = uy
        v[:, -1] = v[:, -2]
    if grid.periodic_y:
        avg = 0.5 * (v[0, :] + v[-1, :])
        v[0, :] = avg
        v[-1, :] = avg
    elif channel_walls:
        v[0, :] = 0.0
        v[-1, :] = 0.0
        u[0, :] = 0.0
        u[-1, :] = 0.0
    else:
        v[0, :] = uy
        v[-1, :] = uy
        u[0, :] = ux
        u[-1, :] = ux


def _solid_faces(solid: np.ndarray):
    """Faces touching a solid cell (``enforce_solid_faces`` masks, PY/core/grid.py:87-94)."""
    su = np.zeros((solid.shape[0], solid.shape[1] + 1), dtype=bool)
    sv = np.zeros((solid.shape[0] + 1, solid.shape[1]), dtype=bool)
    su[:, 1:-1] = solid[:, :-1] | solid[:, 1:]
    su[:, 0], su[:, -1] = solid[:, 0], solid[:, -1]
    sv[1:-1, :] = solid[:-1, :] | solid[1:, :]
    sv[0, :], sv[-1, :] = solid[0, :], solid[-1, :]
    return su, sv


def enforce_solid_faces(u, v, solid, wall) -> None:
    """Solid-touching faces take the interpolated wall velocity; PY/core/grid.py:81-97."""
    su, sv = _solid_faces(solid)
    wu, wv = cell_to_faces(wall)
    u[su] = wu[su]
    v[sv] = wv[sv]


def native_divergence_linf(u, v, grid: Grid, solid) -> float:
    """Max |MAC divergence| over fluid cells; PY/core/grid.py:100-111."""
    div = (u[:, 1:] - u[:, :-1]) / grid.dx + (v[1:, :] - v[:-1, :]) / grid.dy
    fluid = ~solid
    return float(np.max(np.abs(div[fluid]))) if np.any(fluid) else 0.0


def solid_face_leakage(u, v, solid, wall) -> float:
    """Max wall-relative speed on fluid/solid interface faces; PY/core/grid.py:114-131."""
    wu, wv = cell_to_faces(wall)
    iu = np.zeros_like(u, dtype=bool)
    iv = np.zeros_like(v, dtype=bool)
    iu[:, 1:-1] = solid[:, :-1] ^ solid[:, 1:]
    iv[1:-1, :] = solid[:-1, :] ^ solid[1:, :]
    worst = 0.0
    if np.any(iu):
        worst = max(worst, float(np.max(np.abs(u[iu] - wu[iu]))))
    if np.any(iv):
        worst = max(worst, float(np.max(np.abs(v[iv] - wv[iv]))))
    return worst


# --------------------------------------------------------------------------- sampling / advection


def sample_staggered(field_, points, grid: Grid, offset):
    """Bilinear sample with cell-unit origin offset; ``sample_staggered_scalar`` PY/core/interpolation.py:9-52."""
    gx = (points[:, 0] - grid.x0) / grid.dx - offset[0]
    gy = (points[:, 1] - grid.y0) / grid.dy - offset[1]
    gx = np.mod(gx, grid.nx) if grid.periodic_x else np.clip(gx, 0.0, field_.shape[1] - 1.0)
    gy = np.mod(gy, grid.ny) if grid.periodic_y else np.clip(gy, 0.0, field_.shape[0] - 1.0)
    ix0 = np.floor(gx).astype(np.int64)
    iy0 = np.floor(gy).astype(np.int64)
    tx = gx - ix0
    ty = gy - iy0
    ix1 = np.mod(ix0 + 1, grid.nx) if grid.periodic_x else np.minimum(ix0 + 1, field_.shape[1] - 1)
    iy1 = np.mod(iy0 + 1, grid.ny) if grid.periodic_y else np.minimum(iy0 + 1, field_.shape[0] - 1)
    out = (
        (1.0 - tx) * (1.0 - ty) * field_[iy0, ix0]
        + tx * (1.0 - ty) * field_[iy0, ix1]
        + (1.0 - tx) * ty * field_[iy1, ix0]
        + tx * ty * field_[iy1, ix1]
    )
    return np.asarray(out, dtype=field_.dtype)


def sample_vector(vel, points, grid: Grid):
    """Per-component cell-centred sample; ``sample_vector`` PY/core/interpolation.py:67-79."""
    return np.stack([sample_staggered(vel[:, :, c], points, grid, (0.5, 0.5)) for c in range(vel.shape[2])], axis=1)


def rk2_backtrace(vel, points, dt: float, grid: Grid):
    """Midpoint RK2 trace through a frozen field; ``rk2_backtrace`` PY/core/grid.py:527-537."""
    k1 = sample_vector(vel, points, grid)
    mid = points - 0.5 * dt * k1
    k2 = sample_vector(vel, mid, grid)
    return points - dt * k2


def local_velocity_bounds(vel, grid: Grid):
    """3x3 componentwise min/max (clamped or wrapped); PY/core/grid.py:540-569."""
    ny, nx, _ = vel.shape
    rows = np.arange(ny)
    cols = np.arange(nx)
    lo = vel.copy()
    hi = vel.copy()
    for oy in (-1, 0, 1):
        r = np.mod(rows + oy, ny) if grid.periodic_y else np.clip(rows + oy, 0, ny - 1)
        for ox in (-1, 0, 1):
            c = np.mod(cols + ox, nx) if grid.periodic_x else np.clip(cols + ox, 0, nx - 1)
            nb = vel[r[:, None], c[None, :], :]
            lo = np.minimum(lo, nb)
            hi = np.maximum(hi, nb)
    return lo, hi


def advect_velocity(vel, dt: float, grid: Grid, maccormack: bool):
    """Semi-Lagrangian (optionally limited MacCormack) cell advection; PY/core/grid.py:506-524."""
    pts = cell_centers(grid).reshape(-1, 2)
    first = sample_vector(vel, rk2_backtrace(vel, pts, dt, grid), grid).reshape(vel.shape)
    if not maccormack:
        return first
    fwd = sample_vector(first, rk2_backtrace(first, pts, -dt, grid), grid).reshape(vel.shape)
    corrected = first + 0.5 * (vel - fwd)
    lo, hi = local_velocity_bounds(vel, grid)
    lo = np.minimum(lo, first)
    hi = np.maximum(hi, first)
    return np.asarray(np.clip(corrected, lo, hi), dtype=vel.dtype)


def face_positions(grid: Grid):
    """u and v face centres as (P, 2) points in row-major face order; ``_face_positions``
    PY/core/grid.py:306-321 (numpy linspace ends)."""
    u_x = np.linspace(grid.x0, grid.x1, grid.nx + 1)
    u_y = np.linspace(grid.y0 + 0.5 * grid.dy, grid.y1 - 0.5 * grid.dy, grid.ny)
    v_x = np.linspace(grid.x0 + 0.5 * grid.dx, grid.x1 - 0.5 * grid.dx, grid.nx)
    v_y = np.linspace(grid.y0, grid.y1, grid.ny + 1)
    uxx, uyy = np.meshgrid(u_x, u_y)
    vxx, vyy = np.meshgrid(v_x, v_y)
    return np.stack((uxx, uyy), axis=2).reshape(-1, 2), np.stack((vxx, vyy), axis=2).reshape(-1, 2)


def _face_bounds(f):
    """3x3 minimum / maximum with edge padding; ``_face_local_bounds`` PY/core/grid.py:336-347."""
    p = np.pad(f, 1, mode="edge")
    nb = [p[1 + oy:1 + oy + f.shape[0], 1 + ox:1 + ox + f.shape[1]] for oy in (-1, 0, 1) for ox in (-1, 0, 1)]
    return np.minimum.reduce(nb), np.maximum.reduce(nb)


def advect_faces(u, v, dt: float, grid: Grid, maccormack: bool):
    """Face-centred semi-Lagrangian / MacCormack transport; ``advect_faces`` PY/core/grid.py:350-376."""
    vel = faces_to_cell(u, v)
    up, vp = face_positions(grid)
    fu = sample_staggered(u, rk2_backtrace(vel, up, dt, grid), grid, (0.0, 0.5)).reshape(u.shape)
    fv = sample_staggered(v, rk2_backtrace(vel, vp, dt, grid), grid, (0.5, 0.0)).reshape(v.shape)
    if not maccormack:
        return fu, fv
    fwd = faces_to_cell(fu, fv)
    bu = sample_staggered(fu, rk2_backtrace(fwd, up, -dt, grid), grid, (0.0, 0.5)).reshape(u.shape)
    bv = sample_staggered(fv, rk2_backtrace(fwd, vp, -dt, grid), grid, (0.5, 0.0)).reshape(v.shape)
    cu = fu + 0.5 * (u - bu)
    cv = fv + 0.5 * (v - bv)
    lu, hu = _face_bounds(u)
    lv, hv = _face_bounds(v)
    return np.asarray(np.clip(cu, lu, hu), dtype=u.dtype), np.asarray(np.clip(cv, lv, hv), dtype=v.dtype)


def implicit_diffuse_faces(u, v, nu: float, dt: float, grid: Grid, tol: float = 1.0e-5, max_iter: int = 640):
    """Jacobi viscosity on each face array; ``implicit_diffuse_faces`` PY/core/grid.py:276-303."""
    su, iu, ru, cu = _jacobi_component(u, nu, dt, grid, tol, max_iter)
    sv, iv, rv, cv = _jacobi_component(v, nu, dt, grid, tol, max_iter)
    return su, sv, max(iu, iv), max(ru, rv), cu and cv


def centered_derivative(f, h: float, axis: int, periodic: bool, duplicate_endpoint: bool = False):
    """``centered_derivative`` PY/core/grid.py:379-406: periodic centred differences (the duplicated
    endpoint of a periodic face array is rebuilt from the first), else np.gradient edge order 2."""
    if periodic:
        if duplicate_endpoint:
            n = f.shape[axis] - 1
            logical = np.take(f, np.arange(n), axis=axis)
            d = (np.roll(logical, -1, axis=axis) - np.roll(logical, 1, axis=axis)) / (2.0 * h)
            return np.asarray(np.concatenate((d, np.take(d, [0], axis=axis)), axis=axis), dtype=f.dtype)
        return np.asarray((np.roll(f, -1, axis=axis) - np.roll(f, 1, axis=axis)) / (2.0 * h), dtype=f.dtype)
    return np.asarray(np.gradient(f, h, axis=axis, edge_order=2), dtype=f.dtype)


def cross_velocity_on_faces(u, v, grid: Grid):
    """v at u faces and u at v faces; ``_cross_velocity_on_faces`` PY/core/grid.py:409-432."""
    cu = 0.5 * (u[:, :-1] + u[:, 1:])
    cv = 0.5 * (v[:-1, :] + v[1:, :])
    v_on_u = np.empty_like(u)
    v_on_u[:, 1:-1] = 0.5 * (cv[:, :-1] + cv[:, 1:])
    if grid.periodic_x:
        pv = 0.5 * (cv[:, -1] + cv[:, 0])
        v_on_u[:, 0] = pv
        v_on_u[:, -1] = pv
    else:
        v_on_u[:, 0] = cv[:, 0]
        v_on_u[:, -1] = cv[:, -1]
    u_on_v = np.empty_like(v)
    u_on_v[1:-1, :] = 0.5 * (cu[:-1, :] + cu[1:, :])
    if grid.periodic_y:
        pu = 0.5 * (cu[-1, :] + cu[0, :])
        u_on_v[0, :] = pu
        u_on_v[-1, :] = pu
    else:
        u_on_v[0, :] = cu[0, :]
        u_on_v[-1, :] = cu[-1, :]
    return v_on_u, u_on_v


def skew_face_advection_rate(u, v, grid: Grid) -> float:
    """Staggered advection rate of the skew-RK2 CFL; PY/core/grid.py:435-445."""
    vu, uv = cross_velocity_on_faces(u, v, grid)
    ur = np.abs(u) / grid.dx + np.abs(vu) / grid.dy
    vr = np.abs(uv) / grid.dx + np.abs(v) / grid.dy
    return max(float(np.max(ur)), float(np.max(vr)))


def skew_symmetric_convection(u, v, grid: Grid):
    """Half advective plus half conservative convection; PY/core/grid.py:448-481."""
    vu, uv = cross_velocity_on_faces(u, v, grid)
    px, py = grid.periodic_x, grid.periodic_y
    du_dx = centered_derivative(u, grid.dx, 1, px, duplicate_endpoint=px)
    du_dy = centered_derivative(u, grid.dy, 0, py)
    dv_dx = centered_derivative(v, grid.dx, 1, px)
    dv_dy = centered_derivative(v, grid.dy, 0, py, duplicate_endpoint=py)
    adv_u = u * du_dx + vu * du_dy
    adv_v = uv * dv_dx + v * dv_dy
    con_u = centered_derivative(u * u, grid.dx, 1, px, duplicate_endpoint=px) + centered_derivative(vu * u, grid.dy,
                                                                                                    0, py)
    con_v = centered_derivative(uv * v, grid.dx, 1, px) + centered_derivative(v * v, grid.dy, 0, py,
                                                                               duplicate_endpoint=py)
    return (np.asarray(0.5 * (adv_u + con_u), dtype=u.dtype), np.asarray(0.5 * (adv_v + con_v), dtype=v.dtype))


def advect_faces_skew_rk2(u, v, dt: float, grid: Grid, solid, wall, freestream):
    """Explicit midpoint RK2 of skew-symmetric convection; ``advect_faces_skew_rk2``
    PY/core/grid.py:484-503."""
    fu, fv = skew_symmetric_convection(u, v, grid)
    mu = np.asarray(u - 0.5 * dt * fu, dtype=u.dtype)
    mv = np.asarray(v - 0.5 * dt * fv, dtype=v.dtype)
    apply_domain_boundaries(mu, mv, grid, freestream)
    enforce_solid_faces(mu, mv, solid, wall)
    su, sv = skew_symmetric_convection(mu, mv, grid)
    au = np.asarray(u - dt * su, dtype=u.dtype)
    av = np.asarray(v - dt * sv, dtype=v.dtype)
    apply_domain_boundaries(au, av, grid, freestream)
    enforce_solid_faces(au, av, solid, wall)
    return au, av


def advect_scalar(scalar, vel, dt: float, grid: Grid):
    """Semi-Lagrangian transport of a cell scalar by the same RK2 trace.

    No reference counterpart: composed from ``rk2_backtrace`` (PY/core/grid.py:527)
    and ``sample_scalar`` (PY/core/interpolation.py:55-64).
    """
    pts = cell_centers(grid).reshape(-1, 2)
    dep = rk2_backtrace(vel, pts, dt, grid)
    return sample_staggered(scalar, dep, grid, (0.5, 0.5)).reshape(scalar.shape)


# --------------------------------------------------------------------------- viscosity


def _jacobi_component(fld, nu: float, dt: float, grid: Grid, tol: float, max_iter: int):
    """Backward-Euler Jacobi for one component; ``_implicit_diffuse_scalar`` PY/core/grid.py:219-275."""
    if nu <= 0.0:
        return fld.copy(), 0, 0.0, True
    dup_x = grid.periodic_x and fld.shape[1] == grid.nx + 1
    dup_y = grid.periodic_y and fld.shape[0] == grid.ny + 1
    logical = fld[: fld.shape[0] - int(dup_y), : fld.shape[1] - int(dup_x)]
    ax = nu * dt / (grid.dx * grid.dx)
    ay = nu * dt / (grid.dy * grid.dy)
    denom = 1.0 + 2.0 * ax + 2.0 * ay
    orig = logical.copy()
    cur = logical.copy()
    scale = max(float(np.max(np.abs(orig))), 1.0)
    resid = float("inf")
    done = 0
    for it in range(1, max_iter + 1):
        done = it
        if grid.periodic_x:
            left, right = np.roll(cur, 1, axis=1), np.roll(cur, -1, axis=1)
        else:
            left = np.concatenate((cur[:, :1], cur[:, :-1]), axis=1)
            right = np.concatenate((cur[:, 1:], cur[:, -1:]), axis=1)
        if grid.periodic_y:
            down, up = np.roll(cur, 1, axis=0), np.roll(cur, -1, axis=0)
        else:
            down = np.concatenate((cur[:1, :], cur[:-1, :]), axis=0)
            up = np.concatenate((cur[1:, :], cur[-1:, :]), axis=0)
        nxt = (orig + ax * (left + right) + ay * (down + up)) / denom
        resid = float(np.max(np.abs(nxt - cur))) / scale
        cur = nxt
        if resid <= tol:
            break
    out = fld.copy()
    out[: cur.shape[0], : cur.shape[1]] = cur
    if dup_x:
        out[:, -1] = out[:, 0]
    if dup_y:
        out[-1, :] = out[0, :]
    return np.asarray(out, dtype=fld.dtype), done, resid, resid <= tol


def implicit_diffuse(vel, nu: float, dt: float, grid: Grid, tol: float = 1.0e-5, max_iter: int = 640):
    """Per-component Jacobi viscosity; ``implicit_diffuse`` PY/core/grid.py:183-216.

    Returns (velocity, iterations=max over components, residual=max, converged=all).
    """
    comps, iters, resid, ok = [], 0, 0.0, True
    for c in range(vel.shape[2]):
        f, n, r, good = _jacobi_component(vel[:, :, c], nu, dt, grid, tol, max_iter)
        comps.append(f)
        iters = max(iters, n)
        resid = max(resid, r)
        ok = ok and good
    return np.stack(comps, axis=2), iters, resid, ok


# --------------------------------------------------------------------------- pressure


def dst1_ortho(a: np.ndarray, axis: int) -> np.ndarray:
    """Orthonormal DST-I along ``axis`` via the FFT of the odd extension (self-inverse)."""
    n = a.shape[axis]
    moved = np.moveaxis(a, axis, -1)
    ext = np.zeros(moved.shape[:-1] + (2 * (n + 1),), dtype=np.float64)
    ext[..., 1 : n + 1] = moved
    ext[..., n + 2 :] = -moved[..., ::-1]
    spec = np.fft.rfft(ext, axis=-1)
    out = -spec[..., 1 : n + 1].imag / math.sqrt(2.0 * (n + 1))
    return np.moveaxis(out, -1, axis)


def pcg(apply_a, b, apply_m, rtol: float, maxiter: int, callback=None):
    """Preconditioned CG restating ``scipy.sparse.linalg.cg`` (scipy 1.18.0) with x0 = 0, atol = 0.

    Returns (x, info) with info = 0 on convergence and ``maxiter`` when exhausted.
    """
    bnorm = np.linalg.norm(b)
    atol = rtol * float(bnorm)
    if bnorm == 0:
        return b, 0
    x = np.zeros_like(b)
    r = b.copy()
    rho_prev = None
    p = None
    for it in range(maxiter):
        if np.linalg.norm(r) < atol:
            return x, 0
        z = apply_m(r)
        rho = np.dot(r, z)
        if it > 0:
            p *= rho / rho_prev
            p += z
        else:
            p = np.empty_like(r)
            p[:] = z[:]
        q = apply_a(p)
        alpha = rho / np.dot(p, q)
        x += alpha * p
        r -= alpha * q
        rho_prev = rho
        if callback is not None:
            callback(x)
    return x, maxiter


def poisson_operator(fluid: np.ndarray, dx: float, dy: float, periodic_axes=()):
    """Masked negative Laplacian pieces; ``solve_masked_poisson`` PY/core/_scipy_adapter.py:27-70.

    Returns (diagonal, apply) where apply maps a flat pressure to A p.
    """
    ny, nx = fluid.shape
    ix2, iy2 = 1.0 / (dx * dx), 1.0 / (dy * dy)
    diag = np.zeros((ny, nx), dtype=np.float64)
    he = fluid[:, :-1] & fluid[:, 1:]
    ve = fluid[:-1, :] & fluid[1:, :]
    wrap_x = np.zeros(ny, dtype=bool)
    wrap_y = np.zeros(nx, dtype=bool)
    diag[:, :-1] += he * ix2
    diag[:, 1:] += he * ix2
    diag[:-1, :] += ve * iy2
    diag[1:, :] += ve * iy2
    px, py = "x" in periodic_axes, "y" in periodic_axes
    if px:
        wrap_x = fluid[:, -1] & fluid[:, 0]
        diag[:, -1] += wrap_x * ix2
        diag[:, 0] += wrap_x * ix2
    else:
        diag[:, 0] += fluid[:, 0] * ix2
        diag[:, -1] += fluid[:, -1] * ix2
    if py:
        wrap_y = fluid[-1, :] & fluid[0, :]
        diag[-1, :] += wrap_y * iy2
        diag[0, :] += wrap_y * iy2
    else:
        diag[0, :] += fluid[0, :] * iy2
        diag[-1, :] += fluid[-1, :] * iy2
    diag[~fluid] = 1.0

    def apply(flat):
        p = flat.reshape(ny, nx)
        out = diag * p
        out[:, :-1] -= p[:, 1:] * he * ix2
        out[:, 1:] -= p[:, :-1] * he * ix2
        out[:-1, :] -= p[1:, :] * ve * iy2
        out[1:, :] -= p[:-1, :] * ve * iy2
        if px:
            out[:, -1] -= p[:, 0] * wrap_x * ix2
            out[:, 0] -= p[:, -1] * wrap_x * ix2
        if py:
            out[-1, :] -= p[0, :] * wrap_y * iy2
            out[0, :] -= p[-1, :] * wrap_y * iy2
        out[~fluid] = p[~fluid]
        return out.ravel()

    return diag, apply


def solve_masked_poisson(rhs, fluid, dx: float, dy: float, periodic_axes=(), tol: float = 1.0e-5,
                         max_iter: int = 120, record=None):
    """DST-I (or Jacobi) preconditioned CG for the masked Poisson problem.

    Restates ``solve_masked_poisson`` PY/core/_scipy_adapter.py:16-161. Returns
    (pressure, info, iterations, relative_residual). ``record`` (a list) receives
    the recursive residual norm seen at the top of every CG iteration.
    """
    ny, nx = rhs.shape
    diag, apply = poisson_operator(fluid, dx, dy, periodic_axes)
    size = nx * ny
    inv_diag = 1.0 / np.maximum(diag, np.finfo(rhs.dtype).eps)
    if not periodic_axes:
        kx = np.arange(1, nx + 1, dtype=rhs.dtype)
        ky = np.arange(1, ny + 1, dtype=rhs.dtype)
        lam_x = 2.0 * (1.0 - np.cos(np.pi * kx / (nx + 1))) / (dx * dx)
        lam_y = 2.0 * (1.0 - np.cos(np.pi * ky / (ny + 1))) / (dy * dy)
        inv_lam = 1.0 / (lam_y[:, None] + lam_x[None, :])

        def precond(flat):
            r = flat.reshape(ny, nx)
            t = np.where(fluid, r, 0.0)
            t = dst1_ortho(dst1_ortho(t, 1), 0) * inv_lam
            z = np.asarray(dst1_ortho(dst1_ortho(t, 0), 1), dtype=rhs.dtype)
            z[~fluid] = r[~fluid]
            return z.ravel()
    else:

        def precond(flat):
            return inv_diag.ravel() * flat

    b = rhs.copy()
    singular = "x" in periodic_axes and "y" in periodic_axes
    if singular and np.any(fluid):
        b[fluid] -= np.mean(b[fluid])
    b[~fluid] = 0.0
    if not np.isfinite(b).all():
        raise OracleFailure("nonfinite_state", "pressure RHS contains non-finite values")
    if float(np.max(np.abs(b))) > 0.25 * np.sqrt(np.finfo(rhs.dtype).max / max(size, 1)):
        raise OracleFailure("projection_failure", "pressure RHS exceeds the safe CG dot-product range")
    count = [0]

    def check(xk):
        count[0] += 1
        if not np.isfinite(xk).all():
            raise OracleFailure("nonfinite_state", "pressure CG produced a non-finite iterate")

    if record is not None:
        inner_apply_m = precond

        def precond(flat):  # noqa: F811 - wraps to record ||r|| of the iteration
            record.append(float(np.linalg.norm(flat)))
            return inner_apply_m(flat)

    try:
        with np.errstate(over="raise", invalid="raise", divide="raise"):
            x, info = pcg(apply, b.ravel(), precond, 0.9 * tol, max_iter, check)
    except FloatingPointError as err:
        raise OracleFailure("projection_failure", f"pressure CG failed: {err}") from err
    if not np.isfinite(x).all():
        raise OracleFailure("nonfinite_state", "pressure CG produced a non-finite solution")
    p = x.reshape(ny, nx)
    if singular and np.any(fluid):
        p[fluid] -= np.mean(p[fluid])
    res = b.ravel() - apply(x)
    rel = float(np.linalg.norm(res)) / max(float(np.linalg.norm(b.ravel())), float(np.finfo(rhs.dtype).eps))
    return p, int(info), count[0], rel


@dataclass
class IterReport:
    """``IterativeReport`` (PY/core/grid.py:16-22)."""

    criterion: str
    tolerance: float
    iterations: int
    final_residual: float
    converged: bool


def project_faces(u, v, grid: Grid, solid, wall, freestream, dt: float, channel_walls: bool = False,
                  tol: float = 1.0e-5, max_iter: int = 640, keep: dict | None = None):
    """Pressure projection of face velocities; ``project_faces`` PY/core/grid.py:134-180.

    ``keep`` (a dict) receives the pressure and the recursive residual history.
    """
    apply_domain_boundaries(u, v, grid, freestream, channel_walls)
    enforce_solid_faces(u, v, solid, wall)
    div = (u[:, 1:] - u[:, :-1]) / grid.dx + (v[1:, :] - v[:-1, :]) / grid.dy
    fluid = ~solid
    rhs = np.where(fluid, -div / max(dt, 1.0e-12), 0.0)
    hist = [] if keep is not None else None
    p, info, iters, rel = solve_masked_poisson(np.asarray(rhs, dtype=np.float64), fluid, grid.dx, grid.dy,
                                               grid.periodic_axes, tol, max_iter, hist)
    if keep is not None:
        keep["pressure"] = p.copy()
        keep["residual_history"] = hist
    u[:, 1:-1] -= dt * (p[:, 1:] - p[:, :-1]) / grid.dx
    v[1:-1, :] -= dt * (p[1:, :] - p[:-1, :]) / grid.dy
    if grid.periodic_x:
        u[:, 0] -= dt * (p[:, 0] - p[:, -1]) / grid.dx
        u[:, -1] = u[:, 0]
    if grid.periodic_y:
        v[0, :] -= dt * (p[0, :] - p[-1, :]) / grid.dy
        v[-1, :] = v[0, :]
    apply_domain_boundaries(u, v, grid, freestream, channel_walls)
    enforce_solid_faces(u, v, solid, wall)
    return u, v, IterReport("relative-l2", tol, iters, rel, info == 0 and rel <= tol * (1.0 + 1.0e-6))


# --------------------------------------------------------------------------- diagnostics


def diagnostics_values(vel, u, v, grid: Grid, solid, wall, pivot_x: float, chord: float, freestream_u: float):
    """Diagnostic scalars; ``StableFluidsSolver.diagnostics`` PY/solvers/stable_fluids.py:708-738
    with ``PY/core/metrics.py:24-105``."""
    speed2 = np.sum(vel * vel, axis=-1)
    ke = 0.5 * float(np.mean(speed2))
    du_dy = np.gradient(vel[:, :, 0], grid.dy, axis=0)
    dv_dx = np.gradient(vel[:, :, 1], grid.dx, axis=1)
    omega = dv_dx - du_dy
    ens = 0.5 * float(np.mean(omega * omega))
    du_dx = np.gradient(vel[:, :, 0], grid.dx, axis=1)
    dv_dy = np.gradient(vel[:, :, 1], grid.dy, axis=0)
    dv = du_dx + dv_dy
    div_l2 = float(np.sqrt(np.mean(dv * dv)))
    xs = np.linspace(grid.x0 + 0.5 * grid.dx, grid.x1 - 0.5 * grid.dx, grid.nx)
    wake_cols = xs > pivot_x + chord
    if np.any(wake_cols):
        active = freestream_u - vel[:, wake_cols, 0] > 0.1 * abs(freestream_u)
        active &= ~solid[:, wake_cols]
        wake = float(np.count_nonzero(np.any(active, axis=1)) * grid.dy)
    else:
        wake = 0.0
    down = xs > pivot_x
    recirc = (vel[:, down, 0] < 0.0) & ~solid[:, down]
    recirc_area = float(np.count_nonzero(recirc) * grid.dx * grid.dy)
    return {
        "kinetic_energy": ke,
        "enstrophy": ens,
        "divergence_l2": div_l2,
        "divergence_linf": native_divergence_linf(u, v, grid, solid),
        "solid_leakage": solid_face_leakage(u, v, solid, wall),
        "wake_width": wake,
        "recirculation_area": recirc_area,
    }


# --------------------------------------------------------------------------- solver


def surface_forces(u, v, pressure, solid, grid: Grid, nu: float, omega_degrees: float, pivot, freestream,
                   chord: float, reference_speed: float = 1.0) -> dict[str, float]:
    """Surface forces on the solid body. NOT in the reference (it computes no forces): this is
    the FP64 restatement of this library's own definition, the checker for ``fb_forces``.

    Every face between a fluid cell and a solid cell carries the fluid cell's kinematic
    pressure times the face length, pushing into the solid, and the shear
    ``nu (t_fluid - t_wall) / (h / 2)`` times the face length along the face, where t_fluid is
    the fluid cell's centred velocity component along the face and t_wall the rigid wall
    velocity ``omega x (r - pivot)`` at the face centre. Periodic neighbours wrap. The
    coefficients divide the force along / across (+90 deg) the freestream by 0.5 |U|^2 chord."""
    ny, nx = solid.shape
    dx, dy = grid.dx, grid.dy
    om = math.radians(omega_degrees)
    px, py = float(pivot[0]), float(pivot[1])
    u = np.asarray(u, dtype=np.float64)
    v = np.asarray(v, dtype=np.float64)
    uf = 0.5 * (u[:, :-1] + u[:, 1:])
    vf = 0.5 * (v[:-1, :] + v[1:, :])
    fluid = ~solid
    xf = grid.x0 + np.arange(nx + 1, dtype=np.float64) * dx   # x of the vertical faces
    yf = grid.y0 + np.arange(ny + 1, dtype=np.float64) * dy   # y of the horizontal faces
    fx_p = fy_p = fx_v = fy_v = 0.0

    def shifted(arr, di, dj, periodic_y, periodic_x):
        """arr at (i + di, j + dj), False / 0 outside a non-periodic domain."""
        out = np.roll(arr, (-di, -dj), axis=(0, 1))
        if dj and not periodic_x:
            if dj > 0:
                out[:, -1] = False
            else:
                out[:, 0] = False
        if di and not periodic_y:
            if di > 0:
                out[-1, :] = False
            else:
                out[0, :] = False
        return out

    right = fluid & shifted(solid, 0, 1, grid.periodic_y, grid.periodic_x)
    left = fluid & shifted(solid, 0, -1, grid.periodic_y, grid.periodic_x)
    up = fluid & shifted(solid, 1, 0, grid.periodic_y, grid.periodic_x)
    down = fluid & shifted(solid, -1, 0, grid.periodic_y, grid.periodic_x)
    jj = np.broadcast_to(np.arange(nx), (ny, nx))
    ii = np.broadcast_to(np.arange(ny)[:, None], (ny, nx))
    fx_p = float(np.sum(pressure[right]) * dy - np.sum(pressure[left]) * dy)
    fy_p = float(np.sum(pressure[up]) * dx - np.sum(pressure[down]) * dx)
    vw_r = om * (xf[jj[right] + 1] - px)
    vw_l = om * (xf[jj[left]] - px)
    fy_v = float(np.sum(nu * (vf[right] - vw_r) / (0.5 * dx) * dy) + np.sum(nu * (vf[left] - vw_l) / (0.5 * dx) * dy))
    uw_u = -om * (yf[ii[up] + 1] - py)
    uw_d = -om * (yf[ii[down]] - py)
    fx_v = float(np.sum(nu * (uf[up] - uw_u) / (0.5 * dy) * dx) + np.sum(nu * (uf[down] - uw_d) / (0.5 * dy) * dx))
    fx, fy = fx_p + fx_v, fy_p + fy_v
    ux, uy = float(freestream[0]), float(freestream[1])
    speed = math.hypot(ux, uy)
    if speed > 0.0:
        ux, uy = ux / speed, uy / speed
    else:
        ux, uy, speed = 1.0, 0.0, (reference_speed if reference_speed > 0.0 else 1.0)
    q = 0.5 * speed * speed * chord
    return {"pressure_x": fx_p, "pressure_y": fy_p, "viscous_x": fx_v, "viscous_y": fy_v, "force_x": fx,
            "force_y": fy, "drag_coefficient": (fx * ux + fy * uy) / q, "lift_coefficient": (-fx * uy + fy * ux) / q}


def _opt_float(options, name, default):
    value = options.get(name, default)
    if isinstance(value, bool) or not isinstance(value, (int, float)):
        raise TypeError(f"{name} must be numeric")
    return float(value)


def _opt_int(options, name, default):
    value = options.get(name, default)
    if isinstance(value, bool) or not isinstance(value, int):
        raise TypeError(f"{name} must be an integer")
    return value


def _opt_limit(options, name):
    value = options.get(name)
    if value is None:
        return float("inf")
    if isinstance(value, bool) or not isinstance(value, (int, float)):
        raise TypeError(f"{name} must be numeric")
    value = float(value)
    if not np.isfinite(value) or value < 0.0:
        raise ValueError(f"{name} must be finite and non-negative")
    return value


@dataclass
class OracleStep:
    """Per-advance record (mirrors the ``StepReport`` evidence, PY/solvers/stable_fluids.py:576-603)."""

    substeps: int
    max_speed: float
    evidence: dict = field(default_factory=dict)


class OracleSolver:
    """CPU restatement of ``StableFluidsSolver`` (PY/solvers/stable_fluids.py:119-738).

    Covers initialize (:195), restart (:218), the projection guard (:256), advance
    with substep planning, retries, rollback and postconditions (:332-603),
    cell velocity / sampling (:605-611), export (:613), import (:636) and
    diagnostics (:708). Optionally also carries a passive cell scalar advected by
    the velocity trace of each substep (no reference counterpart).
    """

    def __init__(self, scenario, keep_pressure: bool = False):
        self.sc = scenario
        self.grid = Grid.from_domain(scenario.domain)
        self.dtype = np.dtype(np.float32 if scenario.precision == "float32" else np.float64)
        self.opts = dict(scenario.solver_options)
        self.foil = scenario.foil
        self.keep_pressure = keep_pressure
        self.pressure = None
        self.residual_history = []
        self.scalar = None

    # ---- helpers
    def _mask(self, angle):
        return naca_mask(self.foil.naca, self.foil.chord, self.foil.pivot, self.grid, angle)

    def _wall(self, omega):
        return wall_velocity_grid(self.foil.pivot, omega, self.grid)

    @property
    def reference_speed(self):
        fs = float(np.linalg.norm(np.asarray(self.sc.freestream, dtype=np.float64)))
        ic = str(self.opts.get("initial_condition", "freestream"))
        return max(fs, 1.0 if ic in ("taylor-green", "poiseuille") else 0.0, 1.0e-12)

    def _initial_velocity(self):
        """``_initial_velocity`` PY/solvers/stable_fluids.py:102-116."""
        g = self.grid
        vel = np.empty((g.ny, g.nx, 2), dtype=self.dtype)
        vel[...] = np.asarray(self.sc.freestream[:2], dtype=self.dtype)
        ic = str(self.opts.get("initial_condition", "freestream"))
        pos = cell_centers(g)
        if ic == "taylor-green":
            vel[:, :, 0] = np.sin(pos[:, :, 0]) * np.cos(pos[:, :, 1])
            vel[:, :, 1] = -np.cos(pos[:, :, 0]) * np.sin(pos[:, :, 1])
        elif ic == "poiseuille":
            radius = 0.5 * (g.y1 - g.y0)
            center = 0.5 * (g.y0 + g.y1)
            vel[:, :, 0] = 1.5 * (1.0 - ((pos[:, :, 1] - center) / radius) ** 2)
            vel[:, :, 1] = 0.0
        return vel

    # ---- lifecycle
    def initialize(self):
        """``initialize`` PY/solvers/stable_fluids.py:195-216."""
        c0 = self.sc.control_at(0.0)
        self.time = 0.0
        self.angle = c0.angle_degrees
        self.omega = c0.angular_velocity_degrees
        self.reynolds = float(self.sc.reynolds)
        mode = self.opts.get("stable_advection", "maccormack")
        if mode not in ("maccormack", "semi-lagrangian", "skew-rk2"):
            raise ValueError(f"unknown stable_advection {mode}")
        self.maccormack = mode == "maccormack"
        self.skew = mode == "skew-rk2"
        self.face = bool(self.opts.get("stable_face_advection", False))
        self.u, self.v = cell_to_faces(self._initial_velocity())
        self.solid = self._mask(self.angle)
        self.last_projection = IterReport("relative-l2", 0.0, 0, 0.0, True)
        self.last_viscosity = IterReport("update-linf", 0.0, 0, 0.0, True)
        self._project(max(self.sc.output_dt, 1.0e-4))

    def restart(self, time, angle, reynolds):
        """``restart`` PY/solvers/stable_fluids.py:218-236."""
        self.initialize()
        self.reynolds = float(reynolds)
        self.time = float(time)
        self.angle, self.omega = float(angle), 0.0
        self.solid = self._mask(angle)
        vel = self._initial_velocity()
        wall = self._wall(0.0)
        vel[self.solid] = wall[self.solid]
        self.u, self.v = cell_to_faces(vel)
        self._project(max(self.sc.output_dt, 1.0e-4))

    def cell_velocity(self):
        return faces_to_cell(self.u, self.v)

    def _project(self, dt):
        """Projection guard; ``_apply_projection`` PY/solvers/stable_fluids.py:256-330."""
        g = self.grid
        channel = str(self.opts.get("initial_condition", "")) == "poiseuille"
        tol = _opt_float(self.opts, "pressure_tolerance", 1.0e-5)
        max_iter = _opt_int(self.opts, "pressure_max_iterations", 640)
        cfl = float(self.opts.get("stable_cfl", 0.7))
        if getattr(self, "skew", False):
            cfl = min(cfl, 0.4)
        limit = max(1.0, 2.0 * cfl)
        wall = self._wall(self.omega)
        if not all(np.isfinite(a).all() for a in (self.u, self.v, wall)):
            raise OracleFailure("nonfinite_state", "Stable Fluids projection received non-finite velocity",
                                "projection")
        face_speed = max(float(np.max(np.abs(self.u))), float(np.max(np.abs(self.v))))
        wall_speed = float(np.max(np.linalg.norm(wall[self.solid], axis=1))) if np.any(self.solid) else 0.0
        proj_cfl = max(face_speed, wall_speed) * dt / min(g.dx, g.dy)
        if proj_cfl > limit:
            raise OracleFailure("excessive_velocity", "projection CFL exceeded", "projection",
                                {"maximum_cfl": proj_cfl, "maximum_cfl_limit": limit})
        keep = {} if self.keep_pressure else None
        self.u, self.v, rep = project_faces(self.u, self.v, g, self.solid, wall, self.sc.freestream, dt,
                                            channel, tol, max_iter, keep)
        if keep is not None:
            self.pressure = keep["pressure"]
            self.residual_history.append(keep["residual_history"])
        self.last_projection = rep
        if not rep.converged:
            raise OracleFailure("projection_failure", "Stable Fluids pressure CG did not converge", "projection",
                                {"criterion": rep.criterion, "iterations": rep.iterations,
                                 "tolerance": rep.tolerance, "relative_residual": rep.final_residual})
        if not np.isfinite(self.u).all() or not np.isfinite(self.v).all():
            raise OracleFailure("nonfinite_state", "projection produced non-finite velocity", "projection")

    def _snapshot(self):
        return (self.u.copy(), self.v.copy(), self.solid.copy(), self.time, self.angle, self.omega,
                self.last_projection, self.last_viscosity,
                None if self.scalar is None else self.scalar.copy())

    def _restore(self, snap):
        (u, v, s, self.time, self.angle, self.omega, self.last_projection, self.last_viscosity, sc) = snap
        self.u, self.v, self.solid = u.copy(), v.copy(), s.copy()
        self.scalar = None if sc is None else sc.copy()

    def advance(self, control, target_dt: float) -> OracleStep:
        """``advance`` PY/solvers/stable_fluids.py:332-603 (cell-centred transport path)."""
        g = self.grid
        expected = self.time + target_dt
        base = 1.0e-6 if self.sc.precision == "float32" else 1.0e-12
        if abs(control.time - expected) > base * max(1.0, abs(self.time), abs(expected), abs(control.time)):
            raise OracleFailure("time_contract_failure", "control completion time disagrees", "time-mapping")
        cell = self.cell_velocity()
        max_speed = max(float(np.max(np.linalg.norm(cell, axis=2))), abs(self.sc.freestream[0]), 1.0e-6)
        cfl = float(self.opts.get("stable_cfl", 0.7))
        if self.skew:
            cfl = min(cfl, 0.4)
        spacing = min(g.dx, g.dy)
        radius = naca_maximum_radius(self.foil.naca, self.foil.chord)
        wall_speed = abs(np.deg2rad(control.angular_velocity_degrees)) * radius
        sweep = abs(np.deg2rad(control.angle_degrees - self.angle)) * radius / spacing
        rate = skew_face_advection_rate(self.u, self.v, g) if self.skew else max_speed / spacing
        measure = target_dt * rate
        need = max(1.05 * measure / cfl, target_dt * wall_speed / (cfl * spacing), sweep / cfl)
        substeps = max(1, int(np.ceil(need)))
        if substeps > 512:
            raise OracleFailure("stability_limit", "too many internal substeps", "advection" if self.skew else "boundary",
                                {"required_substeps": substeps})
        dt = target_dt / substeps
        nu = self.reference_speed * self.foil.chord / self.reynolds
        div_limit = _opt_limit(self.opts, "mac_maximum_divergence_linf")
        leak_limit = _opt_limit(self.opts, "mac_maximum_solid_leakage")
        vtol = _opt_float(self.opts, "pressure_tolerance", 1.0e-5)
        vmax = _opt_int(self.opts, "pressure_max_iterations", 640)
        snap = self._snapshot()
        start_time, start_angle = self.time, self.angle
        retries = 0
        while True:
            try:
                for k in range(substeps):
                    frac = (k + 1) / substeps
                    sub_time = start_time + frac * target_dt
                    sub_angle = start_angle + frac * (control.angle_degrees - start_angle)
                    if self.skew:
                        sub_wall = self._wall(control.angular_velocity_degrees)
                        au, av = advect_faces_skew_rk2(self.u, self.v, dt, g, self.solid, sub_wall, self.sc.freestream)
                        self.u, self.v, vi, vr, vok = implicit_diffuse_faces(au, av, nu, dt, g, vtol, vmax)
                    elif self.face:
                        au, av = advect_faces(self.u, self.v, dt, g, self.maccormack)
                        self.u, self.v, vi, vr, vok = implicit_diffuse_faces(au, av, nu, dt, g, vtol, vmax)
                    else:
                        vel = faces_to_cell(self.u, self.v)
                        if self.scalar is not None:
                            self.scalar = advect_scalar(self.scalar, vel, dt, g)
                        vel = advect_velocity(vel, dt, g, self.maccormack)
                        vel, vi, vr, vok = implicit_diffuse(vel, nu, dt, g, vtol, vmax)
                        self.u, self.v = cell_to_faces(vel)
                    self.last_viscosity = IterReport("update-linf", vtol, vi, vr, vok)
                    if not vok:
                        raise OracleFailure("convergence_failure", "implicit viscosity did not converge",
                                            "viscosity", {"iterations": vi, "final_residual": vr})
                    self.time, self.angle, self.omega = sub_time, sub_angle, control.angular_velocity_degrees
                    self.solid = self._mask(sub_angle)
                    self._project(dt)
                final = self.cell_velocity()
                if not np.isfinite(final).all():
                    raise OracleFailure("nonfinite_state", "non-finite velocity", "postcondition")
                final_speed = float(np.max(np.linalg.norm(final, axis=2)))
                rate = skew_face_advection_rate(self.u, self.v, g) if self.skew else final_speed / spacing
                accepted = dt * rate
            except Exception:
                self._restore(snap)
                raise
            if accepted <= cfl * (1.0 + 1.0e-6):
                break
            nxt = max(substeps + 1, int(np.ceil(1.05 * substeps * accepted / cfl)))
            self._restore(snap)
            if nxt > 512:
                raise OracleFailure("stability_limit", "retry requires too many substeps", "advection",
                                    {"required_substeps": nxt})
            retries += 1
            substeps = nxt
            dt = target_dt / substeps
        wall = self._wall(control.angular_velocity_degrees)
        div = native_divergence_linf(self.u, self.v, g, self.solid)
        leak = solid_face_leakage(self.u, self.v, self.solid, wall)
        if div > div_limit or leak > leak_limit:
            self._restore(snap)
            raise OracleFailure("postcondition_failure", "MAC postcondition exceeded", "postcondition",
                                {"divergence_linf": div, "solid_leakage": leak})
        self.time = start_time + target_dt
        self.angle = control.angle_degrees
        self.omega = control.angular_velocity_degrees
        return OracleStep(substeps, final_speed, {
            "maximum_fluid_speed": final_speed,
            "maximum_wall_speed": wall_speed,
            "maximum_characteristic_displacement": accepted,
            "maximum_advective_rate": rate,
            "maximum_boundary_sweep": sweep / substeps,
            "stability_retries": retries,
            "pressure_iterations": self.last_projection.iterations,
            "pressure_relative_residual": self.last_projection.final_residual,
            "viscosity_iterations": self.last_viscosity.iterations,
            "viscosity_final_residual": self.last_viscosity.final_residual,
            "divergence_linf": div,
            "solid_leakage": leak,
        })

    def export_velocity(self):
        """Canonical cell velocity with solids zeroed; ``export_state`` PY/solvers/stable_fluids.py:613-634."""
        vel = self.cell_velocity().copy()
        vel[self.solid] = 0.0
        return vel

    def diagnostics(self):
        vel = self.cell_velocity()
        return diagnostics_values(vel, self.u, self.v, self.grid, self.solid, self._wall(self.omega),
                                  self.foil.pivot[0], self.foil.chord, self.sc.freestream[0])
