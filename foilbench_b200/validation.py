"""Entry-point validation shared by the solver lifecycle (reference ``core/solver_validation.py``).

Checks run before any device state is touched, so a rejected call leaves the solver
unchanged, as the reference's transactional contract requires.
"""

from __future__ import annotations

import math

import numpy as np

from foilbench_b200.models import NumericalFailure


def precision_tolerance(precision: str, *values: float) -> float:
    """Absolute time/pose tolerance (solver_validation.py:17-19)."""
    base = 1.0e-6 if precision == "float32" else 1.0e-12
    return base * max(1.0, *(abs(v) for v in values))


def validate_advance_request(current_time: float, control, target_dt: float, precision: str) -> None:
    """Time contract of ``advance`` (solver_validation.py:22-55)."""
    if not math.isfinite(target_dt) or target_dt <= 0.0:
        raise ValueError("target_dt must be finite and positive")
    if not all(math.isfinite(v) for v in (control.time, control.angle_degrees, control.angular_velocity_degrees)):
        raise NumericalFailure("time_contract_failure", "control state must be finite", "time-mapping")
    expected = current_time + target_dt
    tol = precision_tolerance(precision, current_time, expected, control.time)
    if abs(control.time - expected) > tol:
        raise NumericalFailure(
            "time_contract_failure",
            "control completion time disagrees with the requested interval",
            "time-mapping",
            {"expected_time": expected, "control_time": control.time, "target_dt": target_dt},
        )


def validate_restart_state(start) -> None:
    """Restart pose checks (solver_validation.py:58-65)."""
    if not all(math.isfinite(v) for v in (start.time, start.angle_degrees, start.reynolds)):
        raise ValueError("restart state must be finite")
    if start.time < 0.0 or start.reynolds <= 0.0:
        raise ValueError("restart time must be nonnegative and Reynolds positive")


def validate_canonical_import(state, scenario, control, solid: np.ndarray | None) -> None:
    """Canonical import admissibility (solver_validation.py:68-210).

    ``solid`` is the solid mask at the import pose (from the device mask kernel); the
    imported velocity must be exactly zero there.
    """

    def reject(reason, detail, evidence=None):
        raise NumericalFailure(reason, detail, "canonical-import", evidence)

    if state.schema_version not in (1, 2):
        reject("incompatible_domain", "canonical schema version is unsupported")
    if state.dimension != scenario.domain.dimension:
        reject("incompatible_domain", "canonical dimension does not match the scenario")
    if tuple(state.resolution) != tuple(scenario.domain.resolution):
        reject("incompatible_domain", "canonical resolution does not match the scenario")
    if tuple(state.periodic_axes) != tuple(scenario.domain.periodic_axes):
        reject("incompatible_domain", "canonical periodic axes do not match the scenario")
    if state.precision != scenario.precision:
        reject("incompatible_domain", "canonical precision does not match the scenario")
    nz = 1 if state.dimension == 2 else state.resolution[2]
    vshape = (nz, state.resolution[1], state.resolution[0], state.dimension)
    want = np.dtype(state.precision)
    if (
        state.velocity.shape != vshape
        or state.velocity.dtype != want
        or (state.density is not None and (state.density.shape != vshape[:-1] or state.density.dtype != want))
    ):
        reject("incompatible_domain", "canonical array shape or dtype does not match metadata")
    if not np.isfinite(state.velocity).all() or (state.density is not None and not np.isfinite(state.density).all()):
        reject("nonfinite_state", "canonical arrays must be finite at import time")
    sb = np.asarray(state.bounds, dtype=np.float64)
    cb = np.asarray(scenario.domain.bounds, dtype=np.float64)
    tol = precision_tolerance(scenario.precision, *sb.reshape(-1).tolist(), *cb.reshape(-1).tolist())
    if not np.allclose(sb, cb, rtol=0.0, atol=tol):
        reject("incompatible_domain", "canonical bounds do not match the scenario")
    if not all(math.isfinite(v) for v in (control.time, control.angle_degrees, control.angular_velocity_degrees)):
        reject("time_contract_failure", "import control must be finite")
    ctol = precision_tolerance(scenario.precision, state.time, control.time, state.angle_degrees,
                               control.angle_degrees, state.angular_velocity_degrees, control.angular_velocity_degrees)
    if (
        abs(state.time - control.time) > ctol
        or abs(state.angle_degrees - control.angle_degrees) > ctol
        or abs(state.angular_velocity_degrees - control.angular_velocity_degrees) > ctol
    ):
        reject("time_contract_failure", "canonical time or foil control disagrees with the import control",
               {"state_time": state.time, "control_time": control.time, "state_angle": state.angle_degrees,
                "control_angle": control.angle_degrees})
    if state.schema_version == 2 and _foil_key(state.geometry) != _foil_key(scenario.foil):
        reject("incompatible_geometry", "canonical geometry does not match the scenario")
    if state.dimension == 2 and solid is not None:
        cells = state.velocity[0][solid]
        if np.any(cells != 0.0):
            bad = int(np.count_nonzero(np.any(cells != 0.0, axis=1)))
            reject("postcondition_failure", "canonical solid-cell velocity must be exactly zero",
                   {"nonzero_solid_cells": bad})


def _foil_key(foil):
    if foil is None:
        return None
    return (str(foil.naca), float(foil.chord), tuple(float(p) for p in foil.pivot))
