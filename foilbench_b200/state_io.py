"""Canonical flow-state artifacts: ``manifest.json`` + little-endian ``velocity.npy``.

Same on-disk format as the reference (``core/state_io.py:48-190``, contracts
``spec/contracts/canonical-state*.md``): velocity axes (z, y, x, component), C or
Fortran order declared in the manifest, schema versions 1 and 2.
"""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from foilbench_b200.models import CanonicalFlowState, FoilSpec

_SOLVERS = ("stable-fluids", "lbm-d2q9", "pic-flip")
_IMPLEMENTATIONS = ("python", "julia", "typescript", "rust")
_TARGETS = ("native", "node", "browser-worker", "wasm-browser")


def save_canonical_state(state: CanonicalFlowState, directory, build: dict | None = None) -> Path:
    """Write a canonical state directory; ``build`` is informative producer metadata (v2)."""
    out = Path(directory)
    out.mkdir(parents=True, exist_ok=True)
    le = np.dtype(state.precision).newbyteorder("<")
    np.save(out / "velocity.npy", np.ascontiguousarray(np.asarray(state.velocity, dtype=state.precision).astype(le, copy=False)),
            allow_pickle=False)
    if state.density is not None:
        np.save(out / "density.npy",
                np.ascontiguousarray(np.asarray(state.density, dtype=state.precision).astype(le, copy=False)),
                allow_pickle=False)
    manifest: dict[str, object] = {
        "schema_version": state.schema_version,
        "dimension": state.dimension,
        "bounds": [list(b) for b in state.bounds],
        "resolution": list(state.resolution),
        "periodic_axes": list(state.periodic_axes),
        "time": state.time,
        "precision": state.precision,
        "angle_degrees": state.angle_degrees,
        "angular_velocity_degrees": state.angular_velocity_degrees,
        "source_solver": state.source_solver,
        "velocity": {"file": "velocity.npy", "axes": ["z", "y", "x", "component"], "order": "C"},
        "density": None if state.density is None else {"file": "density.npy", "axes": ["z", "y", "x"], "order": "C"},
    }
    if state.schema_version == 1:
        manifest["source_language"] = state.source_language
    else:
        if state.geometry is None or state.producer_execution_target is None:
            raise ValueError("canonical v2 requires geometry and producer target")
        manifest["geometry"] = {"family": "naca-four-digit-v1", "naca": state.geometry.naca,
                                "chord": state.geometry.chord, "pivot": list(state.geometry.pivot)}
        producer: dict[str, object] = {"implementation": state.source_language,
                                       "execution_target": state.producer_execution_target}
        if build is not None:
            producer["build"] = dict(build)
        manifest["producer"] = producer
    (out / "manifest.json").write_text(json.dumps(manifest, indent=2), encoding="utf-8")
    return out


def _check_manifest(m: dict) -> None:
    """Structural checks equivalent to the canonical manifest schemas (v1 and v2)."""
    version = m.get("schema_version")
    if version not in (1, 2):
        raise ValueError("invalid canonical manifest: schema_version must be 1 or 2")
    required = ["schema_version", "dimension", "bounds", "resolution", "periodic_axes", "time", "precision",
                "angle_degrees", "angular_velocity_degrees", "source_solver", "velocity", "density"]
    required += ["source_language"] if version == 1 else ["geometry", "producer"]
    missing = [k for k in required if k not in m]
    if missing:
        raise ValueError(f"invalid canonical manifest: missing {missing}")
    if m["precision"] not in ("float32", "float64"):
        raise ValueError("canonical precision must be float32 or float64")
    if m["source_solver"] not in _SOLVERS:
        raise ValueError("invalid canonical manifest: unknown source_solver")
    if not isinstance(m["time"], (int, float)) or m["time"] < 0:
        raise ValueError("invalid canonical manifest: time")
    if version == 2:
        g = m["geometry"]
        if not isinstance(g, dict) or g.get("family") != "naca-four-digit-v1":
            raise ValueError("invalid canonical manifest: geometry family")
        p = m["producer"]
        if not isinstance(p, dict) or p.get("implementation") not in _IMPLEMENTATIONS or p.get(
                "execution_target") not in _TARGETS:
            raise ValueError("invalid canonical manifest: producer")


def _array_meta(m: dict, name: str, axes: list[str]):
    raw = m.get(name)
    if raw is None:
        return None
    if not isinstance(raw, dict):
        raise TypeError(f"canonical {name} metadata must be an object")
    if raw.get("file") != f"{name}.npy":
        raise ValueError(f"canonical {name} must use {name}.npy")
    if raw.get("axes") != axes:
        raise ValueError(f"canonical {name} axes must be {axes}")
    if raw.get("order") not in ("C", "F"):
        raise ValueError(f"canonical {name} must declare C or Fortran order")
    return raw


def _order_ok(a: np.ndarray, meta: dict) -> bool:
    return bool(a.flags.c_contiguous if meta["order"] == "C" else a.flags.f_contiguous)


def load_canonical_state(directory) -> CanonicalFlowState:
    """Load and validate a canonical state directory (state_io.py:103-187)."""
    src = Path(directory)
    m = json.loads((src / "manifest.json").read_text(encoding="utf-8"))
    if not isinstance(m, dict):
        raise TypeError("manifest.json must contain a JSON object")
    _check_manifest(m)
    vmeta = _array_meta(m, "velocity", ["z", "y", "x", "component"])
    if vmeta is None:
        raise ValueError("canonical velocity metadata is required")
    dmeta = _array_meta(m, "density", ["z", "y", "x"])
    dtype = np.dtype(m["precision"])
    vel = np.load(src / "velocity.npy", allow_pickle=False)
    if vel.dtype != dtype or not _order_ok(vel, vmeta):
        raise ValueError("canonical velocity dtype/order does not match its manifest")
    dens = None
    if dmeta is not None:
        dens = np.load(src / "density.npy", allow_pickle=False)
        if dens.dtype != dtype or not _order_ok(dens, dmeta):
            raise ValueError("canonical density dtype/order does not match its manifest")
    geometry = None
    if isinstance(m.get("geometry"), dict):
        g = m["geometry"]
        geometry = FoilSpec(str(g["naca"]), float(g["chord"]), tuple(float(v) for v in g["pivot"]))
    language = str(m.get("source_language", ""))
    target = None
    if isinstance(m.get("producer"), dict):
        language = str(m["producer"]["implementation"])
        target = str(m["producer"]["execution_target"])
    dim = int(m["dimension"])
    if dim not in (2, 3):
        raise ValueError("canonical dimension must be 2 or 3")
    return CanonicalFlowState(
        schema_version=int(m["schema_version"]),
        dimension=dim,
        bounds=tuple((float(a), float(b)) for a, b in m["bounds"]),
        resolution=tuple(int(n) for n in m["resolution"]),
        periodic_axes=tuple(m["periodic_axes"]),
        time=float(m["time"]),
        precision=m["precision"],
        angle_degrees=float(m["angle_degrees"]),
        angular_velocity_degrees=float(m["angular_velocity_degrees"]),
        source_language=language,
        source_solver=str(m["source_solver"]),
        velocity=np.asarray(vel, dtype=dtype),
        density=None if dens is None else np.asarray(dens, dtype=dtype),
        geometry=geometry,
        producer_execution_target=target,
    )


def midspan_velocity(state: CanonicalFlowState) -> np.ndarray:
    return state.velocity[state.velocity.shape[0] // 2]
