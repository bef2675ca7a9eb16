"""Value types of the solver lifecycle, mirroring the reference's public model objects.

The drop-in solver accepts and returns these types. Field names, meanings and the
validation performed in ``__post_init__`` follow the reference
(``implementations/python/src/foilbench_py/core/models.py``) so code written against
the reference keeps working; objects of the reference's own classes are accepted too
(the solver reads them by attribute).
"""

from __future__ import annotations

import math
from contextvars import ContextVar
from dataclasses import dataclass, field
from typing import Literal, Protocol, runtime_checkable

import numpy as np

Precision = Literal["float32", "float64"]
AxisName = Literal["x", "y", "z"]
ImportStatus = Literal["accepted", "rejected"]
# Failure stage / reason vocabularies (models.py:14-44).
FAILURE_STAGES = (
    "canonical-import", "advection", "viscosity", "projection", "boundary", "collision", "streaming",
    "particle-transfer", "particle-advection", "population-maintenance", "time-mapping", "postcondition",
)
FAILURE_REASONS = (
    "none", "excessive_velocity", "stability_limit", "nonfinite_state", "convergence_failure",
    "incompatible_geometry", "incompatible_domain", "projection_failure", "invalid_density",
    "invalid_population", "invalid_relaxation", "transfer_failure", "postcondition_failure",
    "time_contract_failure", "unsupported_conversion",
)


def _finite(*values: float) -> bool:
    return all(math.isfinite(float(v)) for v in values)


@dataclass(frozen=True, slots=True)
class DomainSpec:
    """Axis-aligned box with a uniform cell resolution (models.py:50-93)."""

    dimension: Literal[2, 3]
    bounds: tuple[tuple[float, float], ...]
    resolution: tuple[int, ...]
    periodic_axes: tuple[AxisName, ...] = ()

    def __post_init__(self) -> None:
        if len(self.bounds) != self.dimension or len(self.resolution) != self.dimension:
            raise ValueError("bounds and resolution must match dimension")
        if any(not _finite(lo, hi) or hi <= lo for lo, hi in self.bounds):
            raise ValueError("each domain upper bound must exceed its lower bound")
        if any(n < 4 for n in self.resolution):
            raise ValueError("each resolution axis must contain at least four cells")
        allowed = ("x", "y") if self.dimension == 2 else ("x", "y", "z")
        if len(set(self.periodic_axes)) != len(self.periodic_axes) or any(a not in allowed for a in self.periodic_axes):
            raise ValueError("periodic axes must be unique and valid for the dimension")

    @property
    def nx(self) -> int:
        return self.resolution[0]

    @property
    def ny(self) -> int:
        return self.resolution[1]

    @property
    def nz(self) -> int:
        return 1 if self.dimension == 2 else self.resolution[2]

    @property
    def dx(self) -> float:
        return (self.bounds[0][1] - self.bounds[0][0]) / self.nx

    @property
    def dy(self) -> float:
        return (self.bounds[1][1] - self.bounds[1][0]) / self.ny


@dataclass(frozen=True, slots=True)
class FoilSpec:
    """NACA four-digit section, chord length and pitch pivot (models.py:96-108)."""

    naca: str
    chord: float
    pivot: tuple[float, ...]

    def __post_init__(self) -> None:
        if len(self.naca) != 4 or not self.naca.isdigit():
            raise ValueError("NACA code must contain exactly four digits")
        if not math.isfinite(self.chord) or self.chord <= 0.0:
            raise ValueError("foil chord must be positive")
        if not self.pivot or not _finite(*self.pivot):
            raise ValueError("foil pivot must contain finite coordinates")


@dataclass(frozen=True, slots=True)
class ControlKeyframe:
    """Angle of attack at a time (models.py:111-120)."""

    time: float
    angle_degrees: float

    def __post_init__(self) -> None:
        if not math.isfinite(self.time) or self.time < 0.0:
            raise ValueError("control keyframe time must be finite and nonnegative")
        if not math.isfinite(self.angle_degrees) or not -90.0 <= self.angle_degrees <= 90.0:
            raise ValueError("control keyframe angle must be finite and within [-90, 90]")


@dataclass(frozen=True, slots=True)
class ControlState:
    """Foil pose at the end of a requested interval (models.py:123-140)."""

    time: float
    angle_degrees: float
    angular_velocity_degrees: float

    def __post_init__(self) -> None:
        if not _finite(self.time, self.angle_degrees, self.angular_velocity_degrees):
            raise ValueError("control state must be finite")
        if self.time < 0.0:
            raise ValueError("control state time cannot be negative")


@dataclass(frozen=True, slots=True)
class Scenario:
    """Declarative scenario (models.py:143-224)."""

    schema_version: int
    id: str
    domain: DomainSpec
    reynolds: float
    freestream: tuple[float, ...]
    foil: FoilSpec
    controls: tuple[ControlKeyframe, ...]
    duration: float
    output_dt: float
    precision: Precision
    seed: int
    solver_options: dict[str, object] = field(default_factory=dict)

    def __post_init__(self) -> None:
        if self.schema_version != 1 or not self.id:
            raise ValueError("scenario schema version and id are required")
        if self.domain.dimension != len(self.freestream):
            raise ValueError("freestream dimensionality must match the domain")
        if len(self.foil.pivot) != self.domain.dimension:
            raise ValueError("foil pivot dimensionality must match the domain")
        if not self.controls:
            raise ValueError("a scenario needs at least one control keyframe")
        if any(b.time <= a.time for a, b in zip(self.controls, self.controls[1:])):
            raise ValueError("control keyframe times must be strictly increasing")
        if not _finite(self.reynolds, self.duration, self.output_dt, *self.freestream):
            raise ValueError("scenario physical values must be finite")
        if self.reynolds <= 0.0 or self.duration <= 0.0 or self.output_dt <= 0.0:
            raise ValueError("Reynolds number, duration, and output_dt must be positive")
        ic = str(self.solver_options.get("initial_condition", "freestream"))
        periodic = set(self.domain.periodic_axes)
        if ic == "taylor-green" and (self.domain.dimension != 2 or periodic != {"x", "y"}):
            raise ValueError("Taylor-Green requires a 2D domain periodic in x and y")
        if ic == "poiseuille" and (self.domain.dimension != 2 or "x" not in periodic or "y" in periodic):
            raise ValueError("Poiseuille requires a 2D domain periodic in x and nonperiodic in y")

    @property
    def dtype(self) -> np.dtype:
        return np.dtype(np.float32 if self.precision == "float32" else np.float64)

    @property
    def reference_speed(self) -> float:
        return reference_speed(self)

    def control_at(self, time: float) -> ControlState:
        return control_at(self.controls, time)


def reference_speed(scenario) -> float:
    """Viscosity speed scale ``max(|U_inf|, prescribed, 1e-12)`` (models.py:196-201)."""
    free = float(np.linalg.norm(np.asarray(scenario.freestream, dtype=np.float64)))
    ic = str(scenario.solver_options.get("initial_condition", "freestream"))
    return max(free, 1.0 if ic in ("taylor-green", "poiseuille") else 0.0, 1.0e-12)


def control_at(controls, time: float) -> ControlState:
    """Smoothstep keyframe interpolation with its time derivative (models.py:203-224)."""
    if len(controls) == 1 or time <= controls[0].time:
        return ControlState(time, controls[0].angle_degrees, 0.0)
    if time >= controls[-1].time:
        return ControlState(time, controls[-1].angle_degrees, 0.0)
    for left, right in zip(controls, controls[1:]):
        if left.time <= time <= right.time:
            span = right.time - left.time
            if span <= 0.0:
                return ControlState(time, right.angle_degrees, 0.0)
            s = (time - left.time) / span
            smooth = s * s * (3.0 - 2.0 * s)
            delta = right.angle_degrees - left.angle_degrees
            return ControlState(time, left.angle_degrees + smooth * delta, 6.0 * s * (1.0 - s) * delta / span)
    return ControlState(time, controls[-1].angle_degrees, 0.0)


@dataclass(frozen=True, slots=True)
class SolverInfo:
    id: str
    display_name: str
    dimensions: tuple[int, ...]
    supports_moving_boundary: bool
    supported_precisions: tuple[str, ...]
    acceleration: str


@dataclass(frozen=True, slots=True)
class InteractiveTuning:
    id: str
    label: str
    value: str | float
    display_value: str
    can_decrease: bool
    can_increase: bool


@dataclass(frozen=True, slots=True)
class StepReport:
    requested_dt: float
    advanced_dt: float
    substeps: int
    max_speed: float
    warnings: tuple[str, ...] = ()
    state_revision: int = 0
    evidence: dict[str, str | int | float | bool] = field(default_factory=dict)


@dataclass(frozen=True, slots=True)
class RestartState:
    time: float
    angle_degrees: float
    reynolds: float


@dataclass(frozen=True, slots=True)
class ReynoldsOutcome:
    requested: float
    effective: float
    warnings: tuple[str, ...] = ()


@dataclass(frozen=True, slots=True)
class ImportReport:
    source_solver: str
    destination_solver: str
    discarded_state: tuple[str, ...]
    warnings: tuple[str, ...] = ()


@dataclass(frozen=True, slots=True)
class ImportOutcome:
    status: ImportStatus
    reason: str
    report: ImportReport | None = None
    warnings: tuple[str, ...] = ()
    stage: str | None = None
    evidence: dict[str, str | int | float | bool] = field(default_factory=dict)

    @property
    def accepted(self) -> bool:
        return self.status == "accepted"


class NumericalFailure(RuntimeError):
    """Classified, anticipated numerical failure (models.py:294-311)."""

    def __init__(self, reason: str, detail: str, stage: str = "postcondition", evidence=None) -> None:
        super().__init__(detail)
        self.reason = reason
        self.stage = stage
        self.evidence = {} if evidence is None else evidence


@dataclass(frozen=True, slots=True)
class Diagnostics:
    values: dict[str, float]
    warnings: tuple[str, ...] = ()
    state_revision: int = 0


# The velocity array whose finiteness the device has already established (the export
# kernel counts non-finite values as it writes the array): CanonicalFlowState then skips its
# own host-side scan of that array, every other check unchanged.
_DEVICE_CHECKED_FINITE: ContextVar[object] = ContextVar("_DEVICE_CHECKED_FINITE", default=None)


@dataclass(frozen=True, slots=True)
class CanonicalFlowState:
    """Portable flow snapshot, velocity axes (z, y, x, component) (models.py:321-391)."""

    schema_version: int
    dimension: Literal[2, 3]
    bounds: tuple[tuple[float, float], ...]
    resolution: tuple[int, ...]
    periodic_axes: tuple[AxisName, ...]
    time: float
    precision: Precision
    angle_degrees: float
    angular_velocity_degrees: float
    source_language: str
    source_solver: str
    velocity: np.ndarray
    density: np.ndarray | None = None
    geometry: FoilSpec | None = None
    producer_execution_target: str | None = None

    def __post_init__(self) -> None:
        if self.schema_version not in (1, 2):
            raise ValueError("unsupported canonical schema version")
        if self.schema_version == 2 and (self.geometry is None or not self.producer_execution_target):
            raise ValueError("canonical v2 requires geometry and producer target identity")
        if len(self.bounds) != self.dimension or len(self.resolution) != self.dimension:
            raise ValueError("canonical bounds and resolution must match dimension")
        if any(not _finite(lo, hi) or hi <= lo for lo, hi in self.bounds):
            raise ValueError("canonical bounds must be finite and increasing")
        if any(n < 1 for n in self.resolution):
            raise ValueError("canonical resolution axes must be positive")
        allowed = ("x", "y") if self.dimension == 2 else ("x", "y", "z")
        if len(set(self.periodic_axes)) != len(self.periodic_axes) or any(a not in allowed for a in self.periodic_axes):
            raise ValueError("canonical periodic axes are invalid for the dimension")
        if not _finite(self.time, self.angle_degrees, self.angular_velocity_degrees):
            raise ValueError("canonical time and control values must be finite")
        if self.time < 0.0:
            raise ValueError("canonical time cannot be negative")
        if not self.source_language or not self.source_solver:
            raise ValueError("canonical source language and solver are required")
        nz = 1 if self.dimension == 2 else self.resolution[2]
        shape = (nz, self.resolution[1], self.resolution[0], self.dimension)
        if self.velocity.shape != shape:
            raise ValueError(f"velocity shape {self.velocity.shape} does not match {shape}")
        if self.density is not None and self.density.shape != shape[:-1]:
            raise ValueError("density shape does not match the canonical grid")
        want = np.dtype(self.precision)
        if self.velocity.dtype != want:
            raise TypeError("velocity dtype does not match canonical precision")
        if self.density is not None and self.density.dtype != want:
            raise TypeError("density dtype does not match canonical precision")
        if _DEVICE_CHECKED_FINITE.get() is not self.velocity and not np.isfinite(self.velocity).all():
            raise ValueError("canonical velocity contains non-finite values")
        if self.density is not None and not np.isfinite(self.density).all():
            raise ValueError("canonical density contains non-finite values")


def scenario_from_dict(raw: dict) -> Scenario:
    """Build a Scenario from a scenario JSON document (field names of ``scenario.schema.json``)."""
    domain = DomainSpec(
        dimension=int(raw["dimension"]),
        bounds=tuple((float(a), float(b)) for a, b in raw["bounds"]),
        resolution=tuple(int(n) for n in raw["resolution"]),
        periodic_axes=tuple(raw.get("periodic_axes", ())),
    )
    foil = raw["foil"]
    return Scenario(
        schema_version=int(raw["schema_version"]),
        id=str(raw["id"]),
        domain=domain,
        reynolds=float(raw["reynolds"]),
        freestream=tuple(float(x) for x in raw["freestream"]),
        foil=FoilSpec(str(foil["naca"]), float(foil["chord"]), tuple(float(x) for x in foil["pivot"])),
        controls=tuple(ControlKeyframe(float(k["time"]), float(k["angle_degrees"])) for k in raw["controls"]),
        duration=float(raw["duration"]),
        output_dt=float(raw["output_dt"]),
        precision=str(raw["precision"]),
        seed=int(raw["seed"]),
        solver_options=dict(raw.get("solver_options", {})),
    )


@runtime_checkable
class FlowSolver(Protocol):
    """Structural solver interface (PY/core/protocol.py:22-57): the members a runner, the
    solver-switching manager and the conformance tests use, so a B200 solver can stand wherever
    the reference's does."""

    info: SolverInfo

    @property
    def reynolds(self) -> float: ...

    @property
    def state_revision(self) -> int: ...

    def initialize(self, scenario: Scenario, geometry, seed: int) -> None: ...

    def restart(self, scenario: Scenario, geometry, seed: int, start: RestartState) -> None: ...

    def set_reynolds(self, reynolds: float) -> ReynoldsOutcome: ...

    def advance(self, control: ControlState, target_dt: float) -> StepReport: ...

    def sample_velocity(self, points: np.ndarray) -> np.ndarray: ...

    def export_state(self) -> CanonicalFlowState: ...

    def import_state(self, state: CanonicalFlowState, control: ControlState) -> ImportOutcome: ...

    def diagnostics(self) -> Diagnostics: ...

    def interactive_tuning(self) -> InteractiveTuning | None: ...

    def adjust_interactive_tuning(self, direction: int) -> InteractiveTuning | None: ...

    def apply_interactive_tuning(self, value: str | float) -> InteractiveTuning | None: ...
