"""Drop-in Stable Fluids solver: the reference ``FlowSolver`` lifecycle on the B200 library.

``StableFluidsSolver`` implements the protocol of ``core/protocol.py:22-57`` with the
semantics of the reference class (``solvers/stable_fluids.py:119-738``): the same
initialisation, restart, Reynolds and transport controls, time contract, transactional
advance/import with classified ``NumericalFailure`` s, canonical export and diagnostics.
Field state lives on the GPU; every numerical stage runs in ``libfoilb200.so``.

Solver options beyond the reference's (``scenario.solver_options``):
  ``pressure_scheme``            "reference" (FP64 CG, the reference's iteration; float32
                                 fields then follow the reference's float32 arithmetic) or
                                 "mixed" (float32 scenarios only: fields and Krylov vectors
                                 stored in FP32, stencils evaluated in FP64, FP32 CG inside
                                 an FP64 defect correction). Default: "reference" for
                                 float64 scenarios, "mixed" for float32 ones.
  ``pressure_fixed_iterations``  run exactly this many CG iterations per projection.
  ``mixed_inner_rtol``           inner FP32 relative residual floor of the mixed scheme (default 3e-6).
  ``pressure_row_transform``     row DST-I of the mixed scheme's preconditioner: "tensor" (TF32
                                 GEMMs on the tensor cores), "fft" (Bluestein FFT) or "auto"
                                 (default: tensor cores on grids of at least 64 tiles of
                                 128 x 128 per parity, else the FFT).
  ``passive_scalar``             carry a cell scalar advected with the velocity trace.
"""

from __future__ import annotations

import ctypes
import math
from typing import Literal

import numpy as np

from foilbench_b200 import _native as N
from foilbench_b200.models import (
    _DEVICE_CHECKED_FINITE,
    CanonicalFlowState,
    ControlState,
    Diagnostics,
    ImportOutcome,
    ImportReport,
    InteractiveTuning,
    NumericalFailure,
    ReynoldsOutcome,
    SolverInfo,
    StepReport,
    reference_speed,
)
from foilbench_b200.validation import validate_advance_request, validate_canonical_import, validate_restart_state

StableTransportMode = Literal["maccormack", "semi-lagrangian", "skew-rk2"]
_MIN_PROJECTION_CFL_LIMIT = 1.0
BUILD_METADATA = {"accelerator": "cuda", "arch": "sm_100a", "library": N.LIB_NAME}


def parse_stable_transport_mode(value: object) -> StableTransportMode:
    if value == "maccormack":
        return "maccormack"
    if value == "semi-lagrangian":
        return "semi-lagrangian"
    if value == "skew-rk2":
        return "skew-rk2"
    raise ValueError(f"unsupported Stable Fluids advection: {value}")


def _float_option(options, name: str, default: float) -> float:
    value = options.get(name, default)
    if isinstance(value, bool) or not isinstance(value, (int, float)):
        raise TypeError(f"{name} must be numeric")
    return float(value)


def _int_option(options, name: str, default: int) -> int:
    value = options.get(name, default)
    if isinstance(value, bool) or not isinstance(value, int):
        raise TypeError(f"{name} must be an integer")
    return value


def _postcondition_limit(options, name: str) -> float:
    value = options.get(name)
    if value is None:
        return float("inf")
    if isinstance(value, bool) or not isinstance(value, (int, float)):
        raise TypeError(f"{name} must be numeric")
    selected = float(value)
    if not np.isfinite(selected) or selected < 0.0:
        raise ValueError(f"{name} must be finite and non-negative")
    return selected


def _cfl_option(options) -> float:
    value = options.get("stable_cfl", 0.7)
    if not isinstance(value, (int, float)):
        raise TypeError("stable_cfl must be numeric")
    return float(value)


_ROW_TRANSFORMS = {"auto": N.ROW_TRANSFORM_AUTO, "fft": N.ROW_TRANSFORM_FFT, "tensor": N.ROW_TRANSFORM_TENSOR}


def pressure_scheme_of(scenario) -> int:
    raw = scenario.solver_options.get("pressure_scheme")
    if raw is None:
        return N.PRESSURE_MIXED if scenario.precision == "float32" else N.PRESSURE_REFERENCE
    if raw == "reference":
        return N.PRESSURE_REFERENCE
    if raw == "mixed":
        if scenario.precision != "float32":
            raise ValueError("pressure_scheme 'mixed' needs a float32 scenario")
        return N.PRESSURE_MIXED
    raise ValueError(f"unsupported pressure_scheme: {raw}")


def scenario_desc(scenario, transport: str = "maccormack") -> N.ScenarioDesc:
    """Resolve a scenario (reference or local value object) into the device description."""
    dom = scenario.domain
    opts = scenario.solver_options
    d = N.ScenarioDesc()
    d.nx, d.ny = int(dom.resolution[0]), int(dom.resolution[1])
    (d.x0, d.x1), (d.y0, d.y1) = (float(dom.bounds[0][0]), float(dom.bounds[0][1])), (
        float(dom.bounds[1][0]), float(dom.bounds[1][1]))
    axes = tuple(dom.periodic_axes)
    d.periodic_x, d.periodic_y = int("x" in axes), int("y" in axes)
    ic = str(opts.get("initial_condition", "freestream"))
    d.channel_walls = int(ic == "poiseuille")
    d.initial_condition = {"taylor-green": N.IC_TAYLOR_GREEN, "poiseuille": N.IC_POISEUILLE}.get(ic, N.IC_FREESTREAM)
    d.freestream_x, d.freestream_y = float(scenario.freestream[0]), float(scenario.freestream[1])
    d.naca = str(scenario.foil.naca).encode("ascii")
    d.chord = float(scenario.foil.chord)
    d.pivot_x, d.pivot_y = float(scenario.foil.pivot[0]), float(scenario.foil.pivot[1])
    d.precision = N.FLOAT32 if scenario.precision == "float32" else N.FLOAT64
    d.pressure_scheme = pressure_scheme_of(scenario)
    d.reference_speed = reference_speed(scenario)
    d.passive_scalar = int(bool(opts.get("passive_scalar", False)))
    d.face_advection = int(bool(opts.get("stable_face_advection", False)))
    rt = str(opts.get("pressure_row_transform", "auto"))
    if rt not in _ROW_TRANSFORMS:
        raise ValueError(f"unsupported pressure_row_transform: {rt}")
    d.row_transform = _ROW_TRANSFORMS[rt]
    apply_runtime_options(d, scenario, transport)
    return d


def apply_runtime_options(d: N.ScenarioDesc, scenario, transport: str) -> None:
    """Options the reference reads at each use (raising TypeError/ValueError before mutation)."""
    opts = scenario.solver_options
    d.cfl = _cfl_option(opts)
    d.pressure_tolerance = _float_option(opts, "pressure_tolerance", 1.0e-5)
    d.pressure_max_iterations = _int_option(opts, "pressure_max_iterations", 640)
    d.pressure_fixed_iterations = _int_option(opts, "pressure_fixed_iterations", 0)
    d.mixed_inner_rtol = _float_option(opts, "mixed_inner_rtol", 0.0)
    d.divergence_limit = _postcondition_limit(opts, "mac_maximum_divergence_linf")
    d.leakage_limit = _postcondition_limit(opts, "mac_maximum_solid_leakage")
    d.advection = {"maccormack": N.ADVECT_MACCORMACK, "skew-rk2": N.ADVECT_SKEW_RK2}.get(transport,
                                                                                    N.ADVECT_SEMI_LAGRANGIAN)


def _failure_from_report(rep: N.Report, message: str, substeps_cap: int = 512) -> NumericalFailure:
    reason, stage = rep.reason_name, rep.stage_name
    ev: dict[str, object] = {}
    if reason == "stability_limit":
        ev = {"required_substeps": int(rep.required_substeps), "maximum_substeps": substeps_cap}
        if rep.stage_name == "advection":
            ev.update({"accepted_measure": rep.accepted_measure, "stability_retries": rep.stability_retries})
        else:
            ev.update({"maximum_fluid_speed": rep.max_speed, "maximum_wall_speed": rep.wall_speed,
                       "boundary_sweep_cells": rep.boundary_sweep})
        message = ("Stable Fluids retry requires too many internal substeps" if rep.stage_name == "advection"
                   else "Stable Fluids motion requires too many internal substeps")
    elif reason == "projection_failure" and stage == "projection":
        ev = {"criterion": "relative-l2", "iterations": int(rep.evidence[0]), "tolerance": rep.evidence[1],
              "relative_residual": rep.evidence[2]}
        message = "Stable Fluids pressure CG did not converge"
    elif reason == "projection_failure":
        message = "pressure CG failed or the pressure RHS exceeds the safe CG dot-product range"
    elif reason == "excessive_velocity":
        ev = {"maximum_cfl": rep.evidence[0], "maximum_cfl_limit": rep.evidence[1]}
        message = f"Stable Fluids projection CFL {rep.evidence[0]:.2f} exceeds {rep.evidence[1]:.2f}"
    elif reason == "postcondition_failure":
        ev = {"divergence_linf": rep.evidence[0], "maximum_divergence_linf": rep.evidence[1],
              "solid_leakage": rep.evidence[2], "maximum_solid_leakage": rep.evidence[3]}
        message = "Stable Fluids exceeded a configured MAC postcondition limit"
    elif reason == "convergence_failure":
        ev = {"criterion": "update-linf", "iterations": rep.viscosity_iterations, "final_residual":
              rep.viscosity_final_residual}
        message = "Stable Fluids implicit viscosity did not converge"
    elif reason == "nonfinite_state":
        message = {"projection": "Stable Fluids projection produced non-finite velocity",
                   "postcondition": "Stable Fluids produced non-finite velocity or pressure"}.get(stage, message)
    return NumericalFailure(reason, message, stage, ev)


class _NativeSolver:
    """Owns one device solver handle."""

    def __init__(self, ctx: N.Context, desc: N.ScenarioDesc):
        self.ctx = ctx
        self.desc = desc
        handle = ctypes.c_void_p()
        N.check(N.lib().fb_solver_create(ctx.handle, ctypes.byref(desc), ctypes.byref(handle)), "fb_solver_create")
        self.handle = handle

    def close(self):
        if self.handle:
            N.lib().fb_solver_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


class StableFluidsSolver:
    """B200 implementation of the Stable Fluids ``FlowSolver``."""

    info = SolverInfo(
        id="stable-fluids",
        display_name="Stable Fluids (MAC, B200)",
        dimensions=(2,),
        supports_moving_boundary=True,
        supported_precisions=("float32", "float64"),
        acceleration="CUDA sm_100a (libfoilb200)",
    )

    def __init__(self, device: int = 0, context: N.Context | None = None) -> None:
        self._ctx = context
        self._device = device
        self._native: _NativeSolver | None = None
        self._scenario = None
        self._geometry = None
        self._control = ControlState(0.0, 0.0, 0.0)
        self._time = 0.0
        self._projection_warning = ""
        self._maccormack = True
        self._skew_rk2 = False
        self._reynolds = 1.0
        self._revision = 0
        self._last_report: N.Report | None = None
        self._last_projection = {"iterations": 0, "relative_residual": 0.0}

    # ------------------------------------------------------------------ protocol properties
    @property
    def reynolds(self) -> float:
        return self._reynolds

    @property
    def state_revision(self) -> int:
        return self._revision

    @property
    def transport_mode(self) -> StableTransportMode:
        if self._skew_rk2:
            return "skew-rk2"
        return "maccormack" if self._maccormack else "semi-lagrangian"

    def set_reynolds(self, reynolds: float) -> ReynoldsOutcome:
        if not np.isfinite(reynolds) or reynolds <= 0.0:
            raise ValueError("Reynolds number must be finite and positive")
        selected = float(reynolds)
        if selected != self._reynolds:
            self._revision += 1
        self._reynolds = selected
        if self._native is not None and self._scenario is not None:
            nu = self._scenario_reference_speed * self._scenario.foil.chord / selected
            N.check(N.lib().fb_set_viscosity(self._native.handle, nu), "fb_set_viscosity")
        return ReynoldsOutcome(self._reynolds, self._reynolds)

    def set_transport_mode(self, mode: StableTransportMode) -> None:
        changed = mode != self.transport_mode
        self._maccormack = mode == "maccormack"
        self._skew_rk2 = mode == "skew-rk2"
        if changed and self._scenario is not None:
            self._revision += 1

    def interactive_tuning(self) -> InteractiveTuning:
        mode = self.transport_mode
        return InteractiveTuning("stable-advection", "adv", mode, mode, mode != "maccormack", mode != "skew-rk2")

    def adjust_interactive_tuning(self, direction: int) -> InteractiveTuning:
        self.set_transport_mode("maccormack" if direction < 0 else "skew-rk2")
        return self.interactive_tuning()

    def apply_interactive_tuning(self, value: str | float) -> InteractiveTuning:
        self.set_transport_mode(parse_stable_transport_mode(value))
        return self.interactive_tuning()

    # ------------------------------------------------------------------ lifecycle
    def _context(self) -> N.Context:
        if self._ctx is None:
            self._ctx = N.default_context(self._device)
        return self._ctx

    def _require(self):
        if self._scenario is None or self._native is None:
            raise RuntimeError("solver has not been initialized")
        return self._scenario, self._native

    def initialize(self, scenario, geometry, seed: int) -> None:
        """``initialize`` (stable_fluids.py:195-216)."""
        del seed
        if scenario.domain.dimension != 2:
            raise NotImplementedError("Stable Fluids Phase 1 supports only 2D")
        mode = parse_stable_transport_mode(scenario.solver_options.get("stable_advection", "maccormack"))
        desc = scenario_desc(scenario, mode)
        if self._native is not None:
            self._native.close()
            self._native = None
        self._scenario = None
        native = _NativeSolver(self._context(), desc)
        control = scenario.control_at(0.0)
        rep = N.Report()
        code = N.lib().fb_initialize(native.handle, float(control.angle_degrees), float(scenario.reynolds),
                                     max(float(scenario.output_dt), 1.0e-4), ctypes.byref(rep))
        if code == N.FB_ERR_NUMERICAL:
            native.close()
            raise _failure_from_report(rep, N.lib().fb_last_error().decode())
        N.check(code, "fb_initialize")
        self._native = native
        self._scenario = scenario
        self._scenario_reference_speed = reference_speed(scenario)
        self._geometry = geometry
        self._control = ControlState(control.time, control.angle_degrees, control.angular_velocity_degrees)
        self._time = 0.0
        self._reynolds = float(scenario.reynolds)
        self._maccormack = mode == "maccormack"
        self._skew_rk2 = mode == "skew-rk2"
        self._last_report = rep
        self._last_projection = {"iterations": rep.pressure_iterations,
                                 "relative_residual": rep.pressure_relative_residual}
        self._revision = 0

    def restart(self, scenario, geometry, seed: int, start) -> None:
        """``restart`` (stable_fluids.py:218-236)."""
        validate_restart_state(start)
        self.initialize(scenario, geometry, seed)
        self.set_reynolds(start.reynolds)
        _, native = self._require()
        rep = N.Report()
        code = N.lib().fb_restart(native.handle, float(start.time), float(start.angle_degrees), float(start.reynolds),
                                  max(float(scenario.output_dt), 1.0e-4), ctypes.byref(rep))
        if code == N.FB_ERR_NUMERICAL:
            raise _failure_from_report(rep, N.lib().fb_last_error().decode())
        N.check(code, "fb_restart")
        self._time = float(start.time)
        self._control = ControlState(start.time, start.angle_degrees, 0.0)
        self._last_report = rep
        self._last_projection = {"iterations": rep.pressure_iterations,
                                 "relative_residual": rep.pressure_relative_residual}
        self._revision = 0

    def advance(self, control: ControlState, target_dt: float) -> StepReport:
        """``advance`` (stable_fluids.py:332-603): substeps, retries and rollback run in the library."""
        native, start_angle = self._prepare_advance(control, target_dt)
        rep = N.Report()
        code = N.lib().fb_advance(native.handle, float(control.time), float(control.angle_degrees),
                                  float(control.angular_velocity_degrees), float(target_dt), ctypes.byref(rep))
        if code == N.FB_ERR_NUMERICAL:
            raise _failure_from_report(rep, N.lib().fb_last_error().decode())
        N.check(code, "fb_advance")
        return self._commit_advance(control, target_dt, rep, start_angle)

    def _prepare_advance(self, control: ControlState, target_dt: float):
        """Argument checks (before any mutation) and the scenario's runtime options."""
        scenario, native = self._require()
        validate_advance_request(self._time, control, target_dt, scenario.precision)
        desc = native.desc
        apply_runtime_options(desc, scenario, self.transport_mode)
        N.check(N.lib().fb_update_options(native.handle, ctypes.byref(desc)), "fb_update_options")
        return native, self._control.angle_degrees

    def _commit_advance(self, control: ControlState, target_dt: float, rep: N.Report, start_angle: float) -> StepReport:
        """Host-side state after an accepted advance, and its StepReport."""
        desc = self._native.desc
        self._time = self._time + target_dt
        self._control = ControlState(self._time, control.angle_degrees, control.angular_velocity_degrees)
        self._revision += 1
        self._last_report = rep
        self._last_projection = {"iterations": rep.pressure_iterations,
                                 "relative_residual": rep.pressure_relative_residual}
        warnings = () if not self._projection_warning else (self._projection_warning,)
        evidence = {
            "maximum_fluid_speed": rep.max_speed,
            "maximum_wall_speed": rep.wall_speed,
            "maximum_characteristic_displacement": rep.accepted_measure,
            "maximum_advective_rate": rep.advective_rate,
            "maximum_boundary_sweep": rep.boundary_sweep,
            "stability_retries": rep.stability_retries,
            "pressure_converged": True,
            "pressure_iterations": rep.pressure_iterations,
            "pressure_relative_residual": rep.pressure_relative_residual,
            "viscosity_converged": bool(rep.viscosity_converged),
            "viscosity_iterations": rep.viscosity_iterations,
            "viscosity_final_residual": rep.viscosity_final_residual,
            "divergence_linf": rep.divergence_linf,
            "solid_leakage": rep.solid_leakage,
            "requested_reynolds": self._reynolds,
            "effective_reynolds": self._reynolds,
            "degraded_motion": rep.wall_speed == 0.0 and abs(control.angle_degrees - start_angle) > 1.0e-9,
            "pressure_outer_iterations": rep.pressure_outer_iterations,
            "pressure_total_iterations": rep.total_pressure_iterations,
            "pressure_scheme": "mixed" if desc.pressure_scheme == N.PRESSURE_MIXED else "reference",
            "device_ms": rep.device_ms,
            "kernel_launches": rep.kernel_launches,
        }
        return StepReport(target_dt, target_dt, rep.substeps, rep.max_speed, warnings, self._revision, evidence)

    # ------------------------------------------------------------------ state access
    def cell_velocity(self) -> np.ndarray:
        scenario, native = self._require()
        out = np.empty((scenario.domain.ny, scenario.domain.nx, 2), dtype=scenario.dtype)
        N.check(N.lib().fb_export_velocity(native.handle, N.ptr(out), out.nbytes, 0), "fb_export_velocity")
        return out

    def face_velocities(self) -> tuple[np.ndarray, np.ndarray]:
        scenario, native = self._require()
        ny, nx = scenario.domain.ny, scenario.domain.nx
        u = np.empty((ny, nx + 1), dtype=scenario.dtype)
        v = np.empty((ny + 1, nx), dtype=scenario.dtype)
        N.check(N.lib().fb_export_faces(native.handle, N.ptr(u), u.nbytes, N.ptr(v), v.nbytes), "fb_export_faces")
        return u, v

    def pressure(self) -> np.ndarray:
        scenario, native = self._require()
        out = np.empty((scenario.domain.ny, scenario.domain.nx), dtype=np.float64)
        N.check(N.lib().fb_export_pressure(native.handle, N.dptr(out), out.nbytes), "fb_export_pressure")
        return out

    def solid_mask(self) -> np.ndarray:
        scenario, native = self._require()
        out = np.empty((scenario.domain.ny, scenario.domain.nx), dtype=np.uint8)
        N.check(N.lib().fb_export_mask(native.handle, N.u8ptr(out), out.size), "fb_export_mask")
        return out.astype(bool)

    def passive_scalar(self) -> np.ndarray:
        scenario, native = self._require()
        out = np.empty((scenario.domain.ny, scenario.domain.nx), dtype=scenario.dtype)
        N.check(N.lib().fb_export_scalar(native.handle, N.ptr(out), out.nbytes), "fb_export_scalar")
        return out

    def set_passive_scalar(self, values: np.ndarray) -> None:
        scenario, native = self._require()
        arr = np.ascontiguousarray(np.asarray(values, dtype=scenario.dtype))
        if arr.shape != (scenario.domain.ny, scenario.domain.nx):
            raise ValueError("passive scalar shape must be (ny, nx)")
        N.check(N.lib().fb_import_scalar(native.handle, N.ptr(arr), arr.nbytes), "fb_import_scalar")

    def sample_velocity(self, points: np.ndarray) -> np.ndarray:
        scenario, native = self._require()
        pts = np.ascontiguousarray(np.asarray(points, dtype=np.float64)[:, :2])
        out = np.empty((pts.shape[0], 2), dtype=np.float64)
        N.check(N.lib().fb_sample_velocity(native.handle, N.dptr(pts), pts.shape[0], N.dptr(out)), "fb_sample_velocity")
        return out.astype(scenario.dtype)

    def export_state(self) -> CanonicalFlowState:
        """Canonical v2 state, solids zeroed (stable_fluids.py:613-634)."""
        scenario, native = self._require()
        vel = N.host_array((scenario.domain.ny, scenario.domain.nx, 2), scenario.dtype)
        bad = ctypes.c_int64(0)
        N.check(N.lib().fb_export_state(native.handle, N.ptr(vel), vel.nbytes, ctypes.byref(bad)), "fb_export_state")
        velocity = vel[None, ...]
        if bad.value != 0:  # the canonical state rejects it (ValueError), as the reference's does
            return self._canonical(scenario, velocity)
        # the device counted no non-finite value as it wrote the array, so the canonical
        # state's finiteness check need not scan it again on the host
        token = _DEVICE_CHECKED_FINITE.set(velocity)
        try:
            return self._canonical(scenario, velocity)
        finally:
            _DEVICE_CHECKED_FINITE.reset(token)

    def _canonical(self, scenario, velocity) -> CanonicalFlowState:
        return CanonicalFlowState(
            schema_version=2,
            dimension=2,
            bounds=tuple(tuple(b) for b in scenario.domain.bounds),
            resolution=tuple(scenario.domain.resolution),
            periodic_axes=tuple(scenario.domain.periodic_axes),
            time=self._time,
            precision=scenario.precision,
            angle_degrees=self._control.angle_degrees,
            angular_velocity_degrees=self._control.angular_velocity_degrees,
            source_language="python",
            source_solver=self.info.id,
            velocity=velocity,
            geometry=scenario.foil,
            producer_execution_target="native",
        )

    def import_state(self, state: CanonicalFlowState, control: ControlState) -> ImportOutcome:
        """``import_state`` (stable_fluids.py:636-706): validate, then re-project on the device."""
        scenario, native = self._require()
        try:
            solid = None
            if state.dimension == 2 and self._geometry is not None:
                from foilbench_b200.geometry import NacaFoil

                solid = NacaFoil(scenario.foil).mask(scenario.domain, control.angle_degrees)
            validate_canonical_import(state, scenario, control, solid)
            velocity = np.ascontiguousarray(np.asarray(state.velocity[0], dtype=scenario.dtype))
            self._apply_import(velocity, state.time, control)
        except NumericalFailure as failure:
            return ImportOutcome("rejected", failure.reason, warnings=(str(failure),), stage=failure.stage,
                                 evidence=failure.evidence)
        self._revision += 1
        report = ImportReport(
            state.source_solver,
            self.info.id,
            ("pressure", "face-centered projection history"),
            ("Stable Fluids rebuilt pressure and face-projection history.",
             *((self._projection_warning,) if self._projection_warning else ())),
        )
        return ImportOutcome("accepted", "none", report, report.warnings)

    def _apply_projection(self, dt: float) -> None:
        """Re-project the current faces at the current pose (the reference's internal projection step)."""
        scenario, native = self._require()
        vel = self.cell_velocity()
        self._apply_import(vel, self._time, self._control, dt)

    def _apply_import(self, velocity: np.ndarray, time: float, control: ControlState, dt: float = 1.0e-4) -> None:
        _, native = self._require()
        rep = N.Report()
        code = N.lib().fb_import_velocity(native.handle, N.ptr(velocity), velocity.nbytes, float(time),
                                          float(control.angle_degrees), float(control.angular_velocity_degrees),
                                          float(dt), ctypes.byref(rep))
        if code == N.FB_ERR_NUMERICAL:
            raise _failure_from_report(rep, N.lib().fb_last_error().decode())
        N.check(code, "fb_import_velocity")
        self._time = float(time)
        self._control = ControlState(control.time, control.angle_degrees, control.angular_velocity_degrees)

    def diagnostics(self) -> Diagnostics:
        """``diagnostics`` (stable_fluids.py:708-738), evaluated on the device."""
        _, native = self._require()
        vals = np.empty(7, dtype=np.float64)
        N.check(N.lib().fb_diagnostics(native.handle, N.dptr(vals), 7), "fb_diagnostics")
        values = {"time": self._time, "requested_reynolds": self._reynolds}
        values.update({name: float(v) for name, v in zip(N.DIAGNOSTIC_NAMES, vals)})
        ordered = {k: values[k] for k in ("time", "requested_reynolds", "kinetic_energy", "enstrophy", "divergence_l2",
                                          "divergence_linf", "solid_leakage", "wake_width", "recirculation_area")}
        warnings = () if not self._projection_warning else (self._projection_warning,)
        if not all(math.isfinite(v) for v in ordered.values()):
            raise NumericalFailure("nonfinite_state", "Stable Fluids produced non-finite diagnostics")
        return Diagnostics(ordered, warnings, self._revision)

    def forces(self) -> dict[str, float]:
        """Surface forces on the foil and their coefficients (FP64, from the current faces and
        the last pressure). The reference computes no forces; the definition is this library's
        (see ``fb_forces`` in include/foilb200.h)."""
        _, native = self._require()
        vals = np.zeros(8, dtype=np.float64)
        N.check(N.lib().fb_forces(native.handle, N.dptr(vals), 8), "fb_forces")
        names = ("pressure_x", "pressure_y", "viscous_x", "viscous_y", "force_x", "force_y", "drag_coefficient",
                 "lift_coefficient")
        return {k: float(v) for k, v in zip(names, vals)}

    # ------------------------------------------------------------------ tuning
    def autotune(self, target_dt: float | None = None, reps: int = 3) -> dict[str, float]:
        """Measure and apply the fastest launch shapes and sweep schedule for this solver's grid
        (fb_autotune): one substep of the current state per candidate, state unchanged. The
        choice is cached for the process, so later solvers of the same grid start from it."""
        scenario, native = self._require()
        dt = float(scenario.output_dt if target_dt is None else target_dt)
        vals = np.zeros(8, dtype=np.float64)
        N.check(N.lib().fb_autotune(native.handle, dt, int(reps), N.dptr(vals), 8), "fb_autotune")
        return {"column_tile": int(vals[0]), "ctas": int(vals[1]), "inner_rtol": float(vals[2]),
                "heuristic_ms": float(vals[3]), "tuned_ms": float(vals[4]), "trials": int(vals[5]),
                "heuristic_column_tile": int(vals[6]), "heuristic_ctas": int(vals[7]),
                "gain": float(vals[3] / vals[4]) if vals[4] > 0 else 1.0}

    def set_launch_shape(self, ctas: int = 0, column_tile: int = 0) -> None:
        """Run the step kernel on `ctas` CTAs with `column_tile`-column tridiagonal tiles (0
        keeps either; fb_set_launch_shape)."""
        _, native = self._require()
        N.check(N.lib().fb_set_launch_shape(native.handle, int(ctas), int(column_tile)), "fb_set_launch_shape")

    def launch_shape(self) -> dict[str, float]:
        """The launch shape in use (CTAs, column tile) and the mixed scheme's inner stop floor."""
        _, native = self._require()
        c, w = ctypes.c_int32(0), ctypes.c_int32(0)
        f = np.zeros(1, dtype=np.float64)
        N.check(N.lib().fb_get_launch_shape(native.handle, ctypes.byref(c), ctypes.byref(w), N.dptr(f)),
                "fb_get_launch_shape")
        return {"ctas": int(c.value), "column_tile": int(w.value), "inner_rtol": float(f[0])}

    # ------------------------------------------------------------------ tracing
    def enable_trace(self, capacity: int = 1 << 16) -> None:
        """Record a device phase trace (CTA 0 timestamps after every grid barrier)."""
        _, native = self._require()
        N.check(N.lib().fb_trace_enable(native.handle, int(capacity)), "fb_trace_enable")
        self._trace_cap = int(capacity)

    def read_trace(self) -> list[tuple[int, int]]:
        _, native = self._require()
        cap = getattr(self, "_trace_cap", 0)
        buf = (ctypes.c_uint64 * max(cap, 1))()
        n = ctypes.c_int64(0)
        N.check(N.lib().fb_trace_read(native.handle, buf, cap, ctypes.byref(n)), "fb_trace_read")
        return [(int(buf[i]) >> 56, int(buf[i]) & ((1 << 56) - 1)) for i in range(min(n.value, cap))]

    @staticmethod
    def trace_summary(entries: list[tuple[int, int]]) -> dict[str, dict[str, float]]:
        """Per-phase device time (us) and count: each stamp's time since the previous stamp."""
        out: dict[str, dict[str, float]] = {}
        prev = None
        for tag, ns in entries:
            if tag != 0 and prev is not None:
                name = N.TRACE_TAGS.get(tag, str(tag))
                d = out.setdefault(name, {"us": 0.0, "count": 0})
                d["us"] += (ns - prev) / 1e3
                d["count"] += 1
            prev = ns
        return out

    def close(self) -> None:
        if self._native is not None:
            self._native.close()
            self._native = None


def solver_ids() -> tuple[str, ...]:
    return ("stable-fluids",)


def create_solver(solver_id: str, device: int = 0):
    """Registry entry point (reference ``solvers/factory.py:15-22``) for the Stable Fluids drop-in."""
    if solver_id == "stable-fluids":
        return StableFluidsSolver(device)
    raise KeyError(f"unknown solver {solver_id!r}; choose from stable-fluids")
