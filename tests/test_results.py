"""Result-v2 artifacts of the drop-in (foilbench_b200/results.py).

CPU: the restated checks are pinned to the reference schema's required fields, constants and
enumerations (tests/golden/result_v2_fields.json, written from the schema by
tests/golden/make_result_v2_fields.py), a consistent row passes and each cross-field rule of
the reference's validate_result_semantics rejects a row that breaks it. GPU: a short scenario
run through the drop-in yields a valid row.
"""

import copy
import json
import math

import pytest

from foilbench_b200 import results as R
from tests._golden import GOLDEN


def test_checks_follow_the_reference_schema():
    f = json.loads((GOLDEN / "result_v2_fields.json").read_text())
    assert list(R.REQUIRED_FIELDS) == f["required"]
    assert f["additional_properties"] is False
    assert f["consts"] == {"schema_version": R.SCHEMA_VERSION, "contract_id": R.CONTRACT_ID,
                           "contract_revision": R.CONTRACT_REVISION}
    assert {k: list(v) for k, v in R.ENUMS.items()} == f["enums"]


def _row():
    steps = [0.010, 0.012, 0.011, 0.030]
    total = sum(steps)
    cells, substeps = 64 * 32, 9
    return {
        "schema_version": 2, "contract_id": "foilbench-phase3-v1", "contract_revision": 5,
        "benchmark_matrix_id": "m", "scenario_id": "s", "repetition": 1, "language": "python",
        "implementation": "python", "execution_target": "native", "solver": "stable-fluids", "git_commit": "x",
        "machine": {}, "precision": "float64", "resolution": [64, 32], "bounds": [[-1.0, 3.0], [-1.0, 1.0]],
        "periodic_axes": [], "reynolds": 100.0, "effective_reynolds": 100.0, "solver_configuration": {},
        "freestream": [1.0, 0.0], "foil": {"naca": "0012", "chord": 1.0, "pivot": [0.0, 0.0]},
        "control_history": [{"time": 0.0, "angle_degrees": 0.0}], "requested_duration": 0.4,
        "simulated_duration": 0.4, "output_dt": 0.1, "seed": 0, "initialization_seconds": 0.1,
        "cold_step_seconds": 0.2, "step_seconds": steps, "median_step_seconds": R._percentile(steps, 0.5),
        "p95_step_seconds": R._percentile(steps, 0.95), "simulated_seconds_per_wall_second": 0.4 / total,
        "cell_updates_per_second": cells * substeps / total, "particle_updates_per_second": 0.0,
        "peak_rss_bytes": 1 << 20, "memory_measurement": "rss", "runtime_startup_seconds": None,
        "worker_startup_seconds": None, "substeps": substeps, "final_state_revision": 5,
        "diagnostic_state_revision": 5, "last_step": {"state_revision": 5}, "diagnostics": {}, "success": True,
        "failure": None, "warnings": [],
    }


def test_consistent_row_passes_and_each_rule_rejects():
    R.validate_result(_row())
    # the percentile is the linear interpolation of the reference
    assert _row()["p95_step_seconds"] == pytest.approx(0.012 + 0.85 * (0.030 - 0.012))
    breaks = [
        ("cell_updates_per_second", lambda r: r.__setitem__("cell_updates_per_second", 1.0)),
        ("stale revision", lambda r: r.__setitem__("diagnostic_state_revision", 4)),
        ("incomplete", lambda r: r.__setitem__("simulated_duration", 0.3)),
        ("failure without evidence", lambda r: r.update(success=False, failure=None)),
        ("rss disagreement", lambda r: r.__setitem__("memory_measurement", "unavailable")),
        ("enum", lambda r: r.__setitem__("solver", "lbm")),
        ("const", lambda r: r.__setitem__("contract_revision", 4)),
        ("extra field", lambda r: r.__setitem__("speed", 1.0)),
        ("missing field", lambda r: r.pop("seed")),
        ("non-finite", lambda r: r["diagnostics"].__setitem__("kinetic_energy", math.inf)),
    ]
    for name, mutate in breaks:
        r = copy.deepcopy(_row())
        mutate(r)
        with pytest.raises(ValueError):
            R.validate_result(r)
        assert name


@pytest.mark.gpu
def test_a_short_run_yields_a_valid_row():
    from dataclasses import replace

    from foilbench_b200.workloads import single

    sc = single("result-v2", 64, 32, "0012", 5.0, 200.0, precision="float32")
    sc = replace(sc, duration=3 * sc.output_dt)
    row = R.run_result(sc, matrix_id="test")
    assert row["success"] is True, row["failure"]
    assert len(row["step_seconds"]) == 3 and row["substeps"] >= 3
    assert row["final_state_revision"] == row["diagnostic_state_revision"] == row["last_step"]["state_revision"]
    assert row["simulated_duration"] == pytest.approx(3 * sc.output_dt)
    assert row["cell_updates_per_second"] > 0.0
    json.dumps(row, allow_nan=False)
