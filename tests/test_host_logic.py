"""Host-side logic of the drop-in that needs no device: model validation, the control
schedule, time contract, canonical artifacts, scenario documents and option parsing.
Mirrors the reference's unit tests of these pieces (tests/unit/test_state_io.py,
test_scenario.py, test_typing_and_models.py)."""

import json
from dataclasses import replace

import numpy as np
import pytest

from foilbench_b200 import _native as N
from foilbench_b200.models import (
    CanonicalFlowState,
    ControlKeyframe,
    ControlState,
    DomainSpec,
    FoilSpec,
    NumericalFailure,
    RestartState,
    Scenario,
    scenario_from_dict,
)
from foilbench_b200.scenario import load_scenario, load_scenario_document
from foilbench_b200.solver import StableFluidsSolver, pressure_scheme_of, scenario_desc
from foilbench_b200.state_io import load_canonical_state, save_canonical_state
from foilbench_b200.validation import validate_advance_request, validate_canonical_import, validate_restart_state


def make(**kw):
    base = dict(schema_version=1, id="t", domain=DomainSpec(2, ((-2.0, 6.0), (-2.0, 2.0)), (48, 24)), reynolds=500.0,
                freestream=(1.0, 0.0), foil=FoilSpec("2412", 1.0, (0.0, 0.0)),
                controls=(ControlKeyframe(0.0, 4.0), ControlKeyframe(1.0, 20.0)), duration=0.05, output_dt=0.01,
                precision="float32", seed=0, solver_options={"stable_advection": "maccormack"})
    base.update(kw)
    return Scenario(**base)


def test_domain_and_foil_validation():
    with pytest.raises(ValueError, match="four cells"):
        DomainSpec(2, ((0.0, 1.0), (0.0, 1.0)), (3, 8))
    with pytest.raises(ValueError, match="upper bound"):
        DomainSpec(2, ((1.0, 0.0), (0.0, 1.0)), (8, 8))
    with pytest.raises(ValueError, match="periodic"):
        DomainSpec(2, ((0.0, 1.0), (0.0, 1.0)), (8, 8), ("x", "x"))
    with pytest.raises(ValueError, match="four digits"):
        FoilSpec("24x2", 1.0, (0.0, 0.0))
    with pytest.raises(ValueError, match="chord"):
        FoilSpec("2412", 0.0, (0.0, 0.0))
    d = DomainSpec(2, ((-1.0, 3.0), (-1.0, 1.0)), (256, 128))
    assert d.dx == 4.0 / 256 and d.dy == 2.0 / 128 and d.nx == 256 and d.ny == 128


def test_scenario_validation_and_control_schedule():
    sc = make()
    c = sc.control_at(0.5)
    assert c.angle_degrees == pytest.approx(12.0)
    assert c.angular_velocity_degrees == pytest.approx(6.0 * 0.25 * 16.0)
    assert sc.control_at(0.0) == ControlState(0.0, 4.0, 0.0)
    assert sc.control_at(2.0) == ControlState(2.0, 20.0, 0.0)
    with pytest.raises(ValueError, match="strictly increasing"):
        make(controls=(ControlKeyframe(1.0, 4.0), ControlKeyframe(1.0, 5.0)))
    with pytest.raises(ValueError, match="Taylor-Green"):
        make(solver_options={"initial_condition": "taylor-green"})
    assert sc.reference_speed == 1.0
    assert make(freestream=(0.0, 0.0), solver_options={}).reference_speed == 1.0e-12


def test_time_contract_and_restart_validation():
    validate_advance_request(0.0, ControlState(0.01, 4.0, 0.0), 0.01, "float32")
    with pytest.raises(ValueError, match="target_dt"):
        validate_advance_request(0.0, ControlState(0.01, 4.0, 0.0), 0.0, "float32")
    with pytest.raises(NumericalFailure) as cap:
        validate_advance_request(0.0, ControlState(1.0, 0.0, 0.0), 0.02, "float64")
    assert cap.value.reason == "time_contract_failure" and cap.value.stage == "time-mapping"
    with pytest.raises(ValueError):
        validate_restart_state(RestartState(-1.0, 0.0, 100.0))


def _state(precision="float32", **kw):
    v = np.arange(1 * 3 * 4 * 2, dtype=precision).reshape(1, 3, 4, 2) / 7.0
    base = dict(schema_version=2, dimension=2, bounds=((0.0, 1.0), (0.0, 1.0)), resolution=(4, 3), periodic_axes=("x",),
                time=0.5, precision=precision, angle_degrees=3.0, angular_velocity_degrees=0.0,
                source_language="python", source_solver="stable-fluids", velocity=v,
                geometry=FoilSpec("0012", 1.0, (0.0, 0.0)), producer_execution_target="native")
    base.update(kw)
    return CanonicalFlowState(**base)


def test_canonical_state_round_trip(tmp_path):
    for version in (1, 2):
        st = _state() if version == 2 else _state(schema_version=1, geometry=None, producer_execution_target=None)
        out = save_canonical_state(st, tmp_path / f"v{version}", build={"arch": "sm_100a"} if version == 2 else None)
        back = load_canonical_state(out)
        assert back.schema_version == version
        np.testing.assert_array_equal(back.velocity, st.velocity)
        assert back.velocity.dtype == np.float32
        assert back.resolution == (4, 3) and back.periodic_axes == ("x",)
        if version == 2:
            assert back.geometry == st.geometry and back.producer_execution_target == "native"
            m = json.loads((out / "manifest.json").read_text())
            assert m["producer"]["build"] == {"arch": "sm_100a"}


def test_canonical_state_rejects_axis_swap_and_bad_order(tmp_path):
    out = save_canonical_state(_state(), tmp_path / "s")
    m = json.loads((out / "manifest.json").read_text())
    m["velocity"]["axes"] = ["z", "x", "y", "component"]
    (out / "manifest.json").write_text(json.dumps(m))
    with pytest.raises(ValueError, match="axes"):
        load_canonical_state(out)
    out2 = save_canonical_state(_state(), tmp_path / "f")
    m = json.loads((out2 / "manifest.json").read_text())
    m["velocity"]["order"] = "F"
    (out2 / "manifest.json").write_text(json.dumps(m))
    with pytest.raises(ValueError, match="order"):
        load_canonical_state(out2)


def test_canonical_state_fortran_layout_loads(tmp_path):
    out = save_canonical_state(_state(), tmp_path / "f")
    vel = np.asfortranarray(np.load(out / "velocity.npy"))
    np.save(out / "velocity.npy", vel)
    m = json.loads((out / "manifest.json").read_text())
    m["velocity"]["order"] = "F"
    (out / "manifest.json").write_text(json.dumps(m))
    back = load_canonical_state(out)
    assert back.velocity.flags.f_contiguous
    assert np.isclose(back.velocity[0, 2, 3, 1], np.float32(23.0 / 7.0))


def test_canonical_import_validation_order():
    sc = make(domain=DomainSpec(2, ((0.0, 1.0), (0.0, 1.0)), (4, 4), ("x",)))
    ctl = ControlState(0.5, 3.0, 0.0)
    v = np.arange(1 * 4 * 4 * 2, dtype=np.float32).reshape(1, 4, 4, 2) / 7.0
    st = _state(resolution=(4, 4), velocity=v)
    validate_canonical_import(replace(st, geometry=sc.foil), sc, ctl, np.zeros((4, 4), bool))
    bad = st.velocity.copy()
    bad[0, 0, 0, 0] = np.nan
    with pytest.raises(NumericalFailure) as cap:
        validate_canonical_import(_raw(st, bad, sc), sc, ctl, None)
    assert cap.value.reason == "nonfinite_state"
    with pytest.raises(NumericalFailure) as cap:
        validate_canonical_import(replace(st, geometry=FoilSpec("0012", 2.0, (0.0, 0.0))), sc, ctl, None)
    assert cap.value.reason == "incompatible_geometry"
    solid = np.zeros((4, 4), bool)
    solid[1, 2] = True
    with pytest.raises(NumericalFailure) as cap:
        validate_canonical_import(replace(st, geometry=sc.foil), sc, ctl, solid)
    assert cap.value.reason == "postcondition_failure" and cap.value.evidence["nonzero_solid_cells"] == 1
    with pytest.raises(NumericalFailure) as cap:
        validate_canonical_import(replace(st, geometry=sc.foil), sc, ControlState(0.7, 3.0, 0.0), None)
    assert cap.value.reason == "time_contract_failure"


def _raw(st, vel, sc):
    # CanonicalFlowState refuses non-finite arrays at construction; mutate after (as the
    # reference test does) to exercise the import-time check.
    good = replace(st, geometry=sc.foil, velocity=st.velocity.copy())
    good.velocity[...] = vel
    return good


def test_scenario_document_loading(tmp_path):
    doc = {"schema_version": 1, "id": "x", "dimension": 2, "bounds": [[-1, 3], [-1, 1]], "resolution": [256, 128],
           "periodic_axes": [], "reynolds": 1000.0, "freestream": [1.0, 0.0],
           "foil": {"naca": "0012", "chord": 1.0, "pivot": [0.0, 0.0]},
           "controls": [{"time": 0.0, "angle_degrees": 8.0}], "duration": 1.0, "output_dt": 0.0078125,
           "precision": "float64", "seed": 0, "solver_options": {"stable_advection": "semi-lagrangian"}}
    (tmp_path / "s.json").write_text(json.dumps(doc))
    sc = load_scenario(tmp_path / "s.json")
    assert sc.domain.resolution == (256, 128) and sc.foil.naca == "0012"
    with pytest.raises(ValueError, match="missing"):
        load_scenario_document({k: v for k, v in doc.items() if k != "foil"})
    assert scenario_from_dict(doc) == sc


def test_device_description_and_options():
    sc = make()
    d = scenario_desc(sc, "maccormack")
    assert (d.nx, d.ny) == (48, 24) and d.naca == b"2412"
    assert d.precision == N.FLOAT32 and d.pressure_scheme == N.PRESSURE_MIXED
    assert d.advection == N.ADVECT_MACCORMACK and d.cfl == 0.7 and d.pressure_max_iterations == 640
    assert d.divergence_limit == float("inf")
    sc64 = make(precision="float64")
    assert pressure_scheme_of(sc64) == N.PRESSURE_REFERENCE
    with pytest.raises(ValueError, match="float32"):
        pressure_scheme_of(make(precision="float64", solver_options={"pressure_scheme": "mixed"}))
    assert pressure_scheme_of(make(solver_options={"pressure_scheme": "reference"})) == N.PRESSURE_REFERENCE
    with pytest.raises(TypeError, match="mac_maximum_divergence_linf"):
        scenario_desc(make(solver_options={"mac_maximum_divergence_linf": "invalid"}))
    with pytest.raises(TypeError, match="pressure_max_iterations"):
        scenario_desc(make(solver_options={"pressure_max_iterations": 1.5}))
    with pytest.raises(ValueError, match="non-negative"):
        scenario_desc(make(solver_options={"mac_maximum_solid_leakage": -1.0}))


def test_uninitialised_solver_and_transport_parsing():
    s = StableFluidsSolver()
    with pytest.raises(RuntimeError, match="not been initialized"):
        s.advance(ControlState(0.01, 0.0, 0.0), 0.01)
    with pytest.raises(ValueError, match="unsupported"):
        s.apply_interactive_tuning("upwind")
    assert s.interactive_tuning().value == "maccormack"
    with pytest.raises(ValueError, match="Reynolds"):
        s.set_reynolds(0.0)
