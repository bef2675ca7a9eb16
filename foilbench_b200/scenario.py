"""Scenario documents (the reference's ``scenario.schema.json`` format).

``load_scenario`` reads a scenario JSON file and checks the fields the schema requires
before constructing the validated ``Scenario`` value object.
"""

from __future__ import annotations

import json
from pathlib import Path

from foilbench_b200.models import Scenario, scenario_from_dict

_REQUIRED = ("schema_version", "id", "dimension", "bounds", "resolution", "periodic_axes", "reynolds", "freestream",
             "foil", "controls", "duration", "output_dt", "precision", "seed")


def validate_scenario_document(raw: dict) -> None:
    if not isinstance(raw, dict):
        raise TypeError("scenario must be a JSON object")
    missing = [k for k in _REQUIRED if k not in raw]
    if missing:
        raise ValueError(f"scenario is missing required fields {missing}")
    if raw["precision"] not in ("float32", "float64"):
        raise ValueError("scenario precision must be float32 or float64")
    if raw["dimension"] not in (2, 3):
        raise ValueError("scenario dimension must be 2 or 3")
    foil = raw["foil"]
    if not isinstance(foil, dict) or not {"naca", "chord", "pivot"} <= set(foil):
        raise ValueError("scenario foil needs naca, chord and pivot")
    if not isinstance(raw["controls"], list) or not raw["controls"]:
        raise ValueError("scenario needs at least one control keyframe")
    if "solver_options" in raw and not isinstance(raw["solver_options"], dict):
        raise ValueError("solver_options must be an object")


def load_scenario_document(raw: dict) -> Scenario:
    validate_scenario_document(raw)
    return scenario_from_dict(raw)


def load_scenario(path) -> Scenario:
    return load_scenario_document(json.loads(Path(path).read_text(encoding="utf-8")))
