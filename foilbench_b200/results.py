"""Result-v2 benchmark artifacts of the drop-in solver.

Restates the reference benchmark runner's timing protocol and result row for one
(scenario, repetition) (``PY/benchmark/runner.py:182-470``), the recorded solver
configuration (``PY/benchmark/artifact.py:9-31``) and the artifact checks
(``spec/schemas/result-v2.schema.json``: required fields, constants and enumerations;
``PY/benchmark/artifact.py:117-174``: the cross-field rules), so that a run of the drop-in
yields rows the reference's tooling accepts:

* ``run_result(scenario, ...)``: a cold solver is initialised and advanced one output
  interval (initialization_seconds, cold_step_seconds), then a fresh solver runs the
  scenario's duration in output intervals, each ``advance`` timed on the host clock
  (step_seconds); diagnostics of the final state; peak resident memory of the process.
* ``validate_result(row)``: raises ``ValueError`` on a row the reference would reject.

The reference runner's optional extras (wake-probe spectrum, recovery window) are not
computed; they are entries of ``diagnostics``, which the schema leaves open.
"""

from __future__ import annotations

import math
import os
import platform
import subprocess
import time
from pathlib import Path
from typing import Callable, Mapping

import numpy as np

SCHEMA_VERSION = 2
CONTRACT_ID = "foilbench-phase3-v1"
CONTRACT_REVISION = 5
REQUIRED_FIELDS = (
    "schema_version", "contract_id", "contract_revision", "benchmark_matrix_id", "scenario_id", "repetition",
    "language", "implementation", "execution_target", "solver", "git_commit", "machine", "precision",
    "resolution", "bounds", "periodic_axes", "reynolds", "effective_reynolds", "solver_configuration",
    "freestream", "foil", "control_history", "requested_duration", "simulated_duration", "output_dt", "seed",
    "initialization_seconds", "cold_step_seconds", "step_seconds", "median_step_seconds", "p95_step_seconds",
    "simulated_seconds_per_wall_second", "cell_updates_per_second", "particle_updates_per_second",
    "peak_rss_bytes", "memory_measurement", "runtime_startup_seconds", "worker_startup_seconds", "substeps",
    "final_state_revision", "diagnostic_state_revision", "last_step", "diagnostics", "success", "failure",
    "warnings",
)
ENUMS = {
    "language": ("python", "julia", "typescript", "rust"),
    "implementation": ("python", "julia", "typescript", "rust"),
    "execution_target": ("native", "node", "browser-worker", "wasm-browser"),
    "solver": ("stable-fluids", "lbm-d2q9", "pic-flip"),
    "precision": ("float32", "float64"),
    "memory_measurement": ("rss", "browser-estimate", "unavailable"),
}
# solver options recorded in every row, with the values a scenario that omits them gets
_SOLVER_OPTION_DEFAULTS: dict[str, object] = {
    "initial_condition": "freestream",
    "stable_advection": "maccormack",
    "stable_face_advection": False,
    "stable_cfl": 0.7,
    "pressure_tolerance": 1.0e-5,
    "pressure_max_iterations": 640,
    "mac_maximum_divergence_linf": None,
    "mac_maximum_solid_leakage": None,
    "pic_flip_blend": 0.95,
    "pic_population_interval": 8,
    "pic_cfl": 0.75,
}


def solver_configuration(scenario) -> dict[str, object]:
    return {name: scenario.solver_options.get(name, default) for name, default in _SOLVER_OPTION_DEFAULTS.items()
            if default is not None or name in scenario.solver_options}


def _percentile(values: list[float], fraction: float) -> float:
    ordered = sorted(values)
    pos = fraction * (len(ordered) - 1)
    lo, hi = math.floor(pos), math.ceil(pos)
    return ordered[lo] + (ordered[hi] - ordered[lo]) * (pos - lo)


def _scalar(value):
    if isinstance(value, np.generic):
        value = value.item()
    if isinstance(value, float) and not math.isfinite(value):
        raise ValueError("benchmark evidence values must be finite")
    return value


def _step_artifact(report) -> dict[str, object] | None:
    if report is None:
        return None
    return {"requested_dt": report.requested_dt, "advanced_dt": report.advanced_dt, "substeps": report.substeps,
            "max_speed": report.max_speed, "state_revision": report.state_revision,
            "evidence": {k: _scalar(v) for k, v in report.evidence.items()}, "warnings": list(report.warnings)}


def _failure_artifact(error: Exception) -> dict[str, object]:
    from foilbench_b200.models import NumericalFailure

    if isinstance(error, NumericalFailure):
        return {"kind": "numerical", "reason": error.reason, "stage": error.stage, "message": str(error),
                "evidence": {k: _scalar(v) for k, v in error.evidence.items()}}
    return {"kind": "exception", "type": type(error).__name__, "message": str(error)}


def _git_commit(root: Path) -> str:
    try:
        out = subprocess.run(["git", "rev-parse", "HEAD"], cwd=root, capture_output=True, text=True, timeout=10)
        return out.stdout.strip() or "unknown"
    except (OSError, subprocess.SubprocessError):
        return "unknown"


def _machine() -> dict[str, object]:
    return {"platform": platform.platform(), "python": platform.python_version(), "processor": platform.processor(),
            "logical_cpus": os.cpu_count(), "numpy": np.__version__, "accelerator": "libfoilb200 (B200, sm_100a)"}


def _rss() -> int | None:
    try:
        import psutil

        return int(psutil.Process().memory_info().rss)
    except Exception:  # noqa: BLE001 - the row then says the measurement is unavailable
        return None


def run_result(scenario, *, matrix_id: str = "foilbench-b200", repetition: int = 1,
               solver_factory: Callable[[], object] | None = None, geometry=None) -> dict[str, object]:
    """One result-v2 row for ``scenario`` (runner.py:206-470, without the optional extras)."""
    from foilbench_b200.geometry import NacaFoil
    from foilbench_b200.solver import StableFluidsSolver

    make = solver_factory or StableFluidsSolver
    geom = geometry if geometry is not None else NacaFoil(scenario.foil)
    init_s = cold_s = 0.0
    elapsed, steps, substeps = 0.0, [], 0
    warnings: list[str] = []
    last, diag_rev, failure, values = None, None, None, {}
    solver = None
    peak = _rss()
    success = True
    try:
        cold = make()
        t0 = time.perf_counter()
        cold.initialize(scenario, geom, scenario.seed)
        init_s = time.perf_counter() - t0
        warm_dt = min(scenario.output_dt, scenario.duration)
        t0 = time.perf_counter()
        cold.advance(scenario.control_at(warm_dt), warm_dt)
        cold_s = time.perf_counter() - t0
        if hasattr(cold, "close"):
            cold.close()
        # a fresh solver, so that the measured run starts from the declared scenario state
        solver = make()
        solver.initialize(scenario, geom, scenario.seed)
        while elapsed < scenario.duration - 1.0e-12:
            dt = min(scenario.output_dt, scenario.duration - elapsed)
            control = scenario.control_at(elapsed + dt)
            t0 = time.perf_counter()
            report = solver.advance(control, dt)
            steps.append(time.perf_counter() - t0)
            last = report
            elapsed += report.advanced_dt
            substeps += report.substeps
            warnings.extend(report.warnings)
            rss = _rss()
            if rss is not None and peak is not None:
                peak = max(peak, rss)
        diagnostics = solver.diagnostics()
        if diagnostics.state_revision != solver.state_revision:
            raise RuntimeError("benchmark diagnostics describe a stale state revision")
        diag_rev = diagnostics.state_revision
        warnings.extend(diagnostics.warnings)
        values = {k: float(v) for k, v in diagnostics.values.items()}
    except Exception as err:  # noqa: BLE001 - a failed run is a row with failure evidence
        success = False
        failure = _failure_artifact(err)
    total = sum(steps)
    cells = math.prod(scenario.domain.resolution)
    particles = values.get("particle_count", 0.0)
    row: dict[str, object] = {
        "schema_version": SCHEMA_VERSION,
        "contract_id": CONTRACT_ID,
        "contract_revision": CONTRACT_REVISION,
        "benchmark_matrix_id": matrix_id,
        "scenario_id": scenario.id,
        "repetition": int(repetition),
        "language": "python",
        "implementation": "python",
        "execution_target": "native",
        "solver": "stable-fluids",
        "git_commit": _git_commit(Path(__file__).resolve().parent),
        "machine": _machine(),
        "precision": scenario.precision,
        "resolution": [int(n) for n in scenario.domain.resolution],
        "bounds": [[float(a), float(b)] for a, b in scenario.domain.bounds],
        "periodic_axes": list(scenario.domain.periodic_axes),
        "reynolds": float(scenario.reynolds),
        "effective_reynolds": float(values.get("effective_reynolds", scenario.reynolds)),
        "solver_configuration": solver_configuration(scenario),
        "freestream": [float(v) for v in scenario.freestream],
        "foil": {"naca": scenario.foil.naca, "chord": scenario.foil.chord, "pivot": list(scenario.foil.pivot)},
        "control_history": [{"time": k.time, "angle_degrees": k.angle_degrees} for k in scenario.controls],
        "requested_duration": float(scenario.duration),
        "simulated_duration": float(elapsed),
        "output_dt": float(scenario.output_dt),
        "seed": int(scenario.seed),
        "initialization_seconds": init_s,
        "cold_step_seconds": cold_s,
        "step_seconds": steps,
        "median_step_seconds": _percentile(steps, 0.5) if steps else 0.0,
        "p95_step_seconds": _percentile(steps, 0.95) if steps else 0.0,
        "simulated_seconds_per_wall_second": elapsed / total if total > 0.0 else 0.0,
        "cell_updates_per_second": cells * substeps / total if total > 0.0 else 0.0,
        "particle_updates_per_second": particles * substeps / total if total > 0.0 else 0.0,
        "peak_rss_bytes": peak,
        "memory_measurement": "rss" if peak is not None else "unavailable",
        "runtime_startup_seconds": None,
        "worker_startup_seconds": None,
        "substeps": int(substeps),
        "final_state_revision": 0 if solver is None else int(solver.state_revision),
        "diagnostic_state_revision": diag_rev,
        "last_step": _step_artifact(last),
        "diagnostics": values,
        "success": success,
        "failure": failure,
        "warnings": sorted(set(warnings)),
    }
    if solver is not None and hasattr(solver, "close"):
        solver.close()
    validate_result(row)
    return row


def _finite_everywhere(value, path="result") -> None:
    if isinstance(value, float) and not math.isfinite(value):
        raise ValueError(f"{path} is not finite")
    if isinstance(value, Mapping):
        for k, v in value.items():
            _finite_everywhere(v, f"{path}.{k}")
    elif isinstance(value, (list, tuple)):
        for i, v in enumerate(value):
            _finite_everywhere(v, f"{path}[{i}]")


def validate_result(row: Mapping[str, object]) -> None:
    """The schema's required fields, constants and enumerations, then the cross-field rules
    of the reference's ``validate_result_semantics`` (artifact.py:117-174)."""
    missing = [k for k in REQUIRED_FIELDS if k not in row]
    if missing:
        raise ValueError(f"result lacks required fields {missing}")
    extra = [k for k in row if k not in REQUIRED_FIELDS]
    if extra:
        raise ValueError(f"result has fields outside the schema {extra}")
    for key, want in (("schema_version", SCHEMA_VERSION), ("contract_id", CONTRACT_ID),
                      ("contract_revision", CONTRACT_REVISION)):
        if row[key] != want:
            raise ValueError(f"{key} must be {want!r}")
    for key, allowed in ENUMS.items():
        if row[key] not in allowed:
            raise ValueError(f"{key} {row[key]!r} is not one of {allowed}")
    if any(int(n) < 4 for n in row["resolution"]) or int(row["repetition"]) < 1:
        raise ValueError("resolution entries must be >= 4 and repetition >= 1")
    for key in ("simulated_duration", "initialization_seconds", "cold_step_seconds", "median_step_seconds",
                "p95_step_seconds", "simulated_seconds_per_wall_second", "cell_updates_per_second",
                "particle_updates_per_second"):
        if float(row[key]) < 0.0:
            raise ValueError(f"{key} must be non-negative")
    if any(float(s) < 0.0 for s in row["step_seconds"]):
        raise ValueError("step_seconds must be non-negative")
    foil = row["foil"]
    if not all(k in foil for k in ("naca", "chord", "pivot")):
        raise ValueError("foil needs naca, chord and pivot")
    _finite_everywhere(dict(row))
    success, failure, last = row["success"], row["failure"], row["last_step"]
    final_rev, diag_rev = int(row["final_state_revision"]), row["diagnostic_state_revision"]
    steps = [float(s) for s in row["step_seconds"]]
    requested, simulated = float(row["requested_duration"]), float(row["simulated_duration"])
    tol = (1.0e-6 if row["precision"] == "float32" else 1.0e-12) * max(1.0, abs(requested))
    if success:
        if failure is not None or not isinstance(last, Mapping) or not steps:
            raise ValueError("successful benchmark result lacks completed-step semantics")
        if diag_rev != final_rev or last.get("state_revision") != final_rev:
            raise ValueError("successful benchmark result contains stale revision evidence")
        if abs(simulated - requested) > tol:
            raise ValueError("successful benchmark result did not complete requested duration")
    elif not isinstance(failure, Mapping):
        raise ValueError("failed benchmark result lacks structured failure evidence")
    if steps:
        total = sum(steps)
        cells = math.prod(int(n) for n in row["resolution"])
        substeps = int(row["substeps"])
        particles = float(row["diagnostics"].get("particle_count", 0.0))
        expected = {
            "median_step_seconds": _percentile(steps, 0.5),
            "p95_step_seconds": _percentile(steps, 0.95),
            "simulated_seconds_per_wall_second": simulated / total,
            "cell_updates_per_second": cells * substeps / total,
            "particle_updates_per_second": particles * substeps / total,
        }
        for key, want in expected.items():
            if not math.isclose(float(row[key]), want, rel_tol=1.0e-10, abs_tol=1.0e-12):
                raise ValueError(f"benchmark result contains inconsistent derived field {key}")
    if (row["memory_measurement"] == "unavailable") != (row["peak_rss_bytes"] is None):
        raise ValueError("memory measurement kind and RSS value disagree")
