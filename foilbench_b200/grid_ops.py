"""Reference-named MAC grid operators evaluated by the device kernels.

Each function runs one stage of the B200 step on caller arrays through the operator
entry points of ``libfoilb200.so`` (the same device code the solver runs), with the
signature and return convention of the reference function it names:

* ``advect_velocity``      <- ``core/grid.py:506``
* ``implicit_diffuse``     <- ``core/grid.py:183``
* ``solve_masked_poisson`` <- ``core/_scipy_adapter.py:16``
* ``project_faces``        <- ``core/grid.py:134``
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from foilbench_b200 import _native as N
from foilbench_b200.models import NumericalFailure


@dataclass(frozen=True, slots=True)
class IterativeReport:
    """``IterativeReport`` (core/grid.py:16-22)."""

    criterion: str
    tolerance: float
    iterations: int
    final_residual: float
    converged: bool


def _desc(domain, precision: str, scheme: int = N.PRESSURE_REFERENCE, tol: float = 1.0e-5, max_iter: int = 640):
    d = N.ScenarioDesc()
    d.nx, d.ny = int(domain.resolution[0]), int(domain.resolution[1])
    (d.x0, d.x1), (d.y0, d.y1) = domain.bounds[0], domain.bounds[1]
    axes = tuple(domain.periodic_axes)
    d.periodic_x, d.periodic_y = int("x" in axes), int("y" in axes)
    d.naca = b"0012"
    d.chord = 1.0
    d.precision = N.FLOAT32 if precision == "float32" else N.FLOAT64
    d.pressure_scheme = scheme
    d.pressure_tolerance = tol
    d.pressure_max_iterations = max_iter
    d.cfl = 0.7
    d.reference_speed = 1.0
    d.divergence_limit = float("inf")
    d.leakage_limit = float("inf")
    return d


def _precision_of(a: np.ndarray) -> str:
    return "float32" if a.dtype == np.float32 else "float64"


def advect_velocity(velocity: np.ndarray, dt: float, domain, maccormack: bool) -> np.ndarray:
    vel = np.ascontiguousarray(velocity)
    out = np.empty_like(vel)
    ctx = N.default_context()
    N.check(N.lib().fb_op_advect_velocity(ctx.handle, ctypes.byref(_desc(domain, _precision_of(vel))), N.ptr(vel),
                                          N.ptr(out), float(dt), int(bool(maccormack))), "fb_op_advect_velocity")
    return out


def implicit_diffuse(velocity: np.ndarray, viscosity: float, dt: float, domain, tolerance: float = 1.0e-5,
                     max_iterations: int = 640):
    vel = np.ascontiguousarray(velocity)
    out = np.empty_like(vel)
    rep = N.Report()
    ctx = N.default_context()
    N.check(N.lib().fb_op_implicit_diffuse(ctx.handle, ctypes.byref(_desc(domain, _precision_of(vel))), N.ptr(vel),
                                           N.ptr(out), float(viscosity), float(dt), float(tolerance),
                                           int(max_iterations), ctypes.byref(rep)), "fb_op_implicit_diffuse")
    return out, IterativeReport("update-linf", tolerance, rep.viscosity_iterations, rep.viscosity_final_residual,
                                bool(rep.viscosity_converged))


class _Domain:
    def __init__(self, nx, ny, dx, dy, periodic_axes):
        self.resolution = (nx, ny)
        self.bounds = ((0.0, dx * nx), (0.0, dy * ny))
        self.periodic_axes = tuple(periodic_axes)


def solve_masked_poisson(rhs: np.ndarray, fluid: np.ndarray, dx: float, dy: float, periodic_axes=(),
                         tolerance: float = 1.0e-5, max_iterations: int = 120, scheme: str = "reference",
                         fixed_iterations: int = 0, row_transform: str = "auto"):
    """Returns (pressure, info, iterations, relative_residual) like the reference adapter.
    ``fixed_iterations`` > 0 runs exactly that many CG iterations whatever the residual (the
    ``pressure_fixed_iterations`` sweep rule); the solve then counts as converged.
    ``row_transform`` ("auto", "fft", "tensor") selects the mixed scheme's preconditioner row DST."""
    ny, nx = rhs.shape
    dom = _Domain(nx, ny, dx, dy, periodic_axes)
    sch = N.PRESSURE_MIXED if scheme == "mixed" else N.PRESSURE_REFERENCE
    d = _desc(dom, "float32" if sch == N.PRESSURE_MIXED else "float64", sch, tolerance, max_iterations)
    d.pressure_fixed_iterations = int(fixed_iterations)
    d.row_transform = {"auto": N.ROW_TRANSFORM_AUTO, "fft": N.ROW_TRANSFORM_FFT,
                       "tensor": N.ROW_TRANSFORM_TENSOR}[row_transform]
    d.x1 = d.x0 + dx * nx
    d.y1 = d.y0 + dy * ny
    b = np.ascontiguousarray(np.asarray(rhs, dtype=np.float64))
    f = np.ascontiguousarray(np.asarray(fluid, dtype=np.uint8))
    p = np.empty_like(b)
    rep = N.Report()
    ctx = N.default_context()
    code = N.lib().fb_op_solve_masked_poisson(ctx.handle, ctypes.byref(d), N.dptr(b), N.u8ptr(f), N.dptr(p),
                                              ctypes.byref(rep))
    if code == N.FB_ERR_NUMERICAL:
        if rep.reason_name == "nonfinite_state":
            raise NumericalFailure("nonfinite_state", "pressure RHS contains non-finite values")
        raise NumericalFailure("projection_failure", "pressure RHS exceeds the safe CG dot-product range")
    N.check(code, "fb_op_solve_masked_poisson")
    info = 0 if rep.pressure_converged else int(max_iterations)
    return p, info, rep.pressure_iterations, rep.pressure_relative_residual


def project_faces(u, v, domain, solid, omega_degrees: float, freestream, dt: float,
                  channel_walls: bool = False, pressure_tolerance: float = 1.0e-5,
                  pressure_max_iterations: int = 640, scheme: str = "reference"):
    """Projection with domain boundaries for ``freestream`` and a rigidly rotating wall
    (angular velocity ``omega_degrees`` about the origin); returns (u, v, IterativeReport)."""
    uu = np.ascontiguousarray(u).copy()
    vv = np.ascontiguousarray(v).copy()
    prec = _precision_of(uu)
    sch = N.PRESSURE_MIXED if scheme == "mixed" else N.PRESSURE_REFERENCE
    d = _desc(domain, prec, sch, pressure_tolerance, pressure_max_iterations)
    d.freestream_x, d.freestream_y = float(freestream[0]), float(freestream[1])
    d.channel_walls = int(bool(channel_walls))
    s = np.ascontiguousarray(np.asarray(solid, dtype=np.uint8))
    rep = N.Report()
    ctx = N.default_context()
    code = N.lib().fb_op_project_faces(ctx.handle, ctypes.byref(d), N.ptr(uu), N.ptr(vv), N.u8ptr(s),
                                       float(omega_degrees), float(dt), ctypes.byref(rep))
    if code == N.FB_ERR_NUMERICAL and rep.reason_name == "projection_failure" and rep.stage_name == "projection":
        return uu, vv, IterativeReport("relative-l2", pressure_tolerance, rep.pressure_iterations,
                                       rep.pressure_relative_residual, False)
    N.check(code, "fb_op_project_faces")
    return uu, vv, IterativeReport("relative-l2", pressure_tolerance, rep.pressure_iterations,
                                   rep.pressure_relative_residual, bool(rep.pressure_converged))
