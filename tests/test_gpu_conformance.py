"""Lifecycle conformance of the B200 Stable Fluids solver, following the reference's own solver
conformance checks (tests/conformance/test_solvers.py in the Python implementation): protocol
and canonical export, transactional imports and failures, argument checks before mutation,
restart, Reynolds changes, pressure budget and determinism."""

from dataclasses import replace

import numpy as np
import pytest

from foilbench_b200 import workloads
from foilbench_b200.geometry import NacaFoil
from foilbench_b200.models import (ControlKeyframe, ControlState, DomainSpec, FlowSolver, FoilSpec, NumericalFailure,
                                   RestartState, Scenario)
from foilbench_b200.solver import StableFluidsSolver, create_solver

pytestmark = pytest.mark.gpu


def _scenario(nx=32, ny=16, precision="float32", **opts):
    return workloads.single("conf", nx, ny, "2412", 8.0, 500.0, precision=precision, tolerance=1e-5,
                            transport="maccormack", extra=opts or None)


def _same_state(a, b):
    assert a.time == b.time and a.angle_degrees == b.angle_degrees
    assert a.angular_velocity_degrees == b.angular_velocity_degrees
    np.testing.assert_array_equal(a.velocity, b.velocity)


def _started(sc):
    s = StableFluidsSolver()
    s.initialize(sc, NacaFoil(sc.foil), sc.seed)
    return s


def test_protocol_and_canonical_export():
    sc = _scenario(64, 32)
    s = create_solver("stable-fluids")
    assert isinstance(s, FlowSolver)
    s.initialize(sc, NacaFoil(sc.foil), sc.seed)
    rep = s.advance(sc.control_at(0.01), 0.01)
    sampled = s.sample_velocity(np.asarray([[-0.5, 0.0], [1.0, 0.5]], dtype=np.float32))
    state = s.export_state()
    diag = s.diagnostics()
    assert rep.advanced_dt == pytest.approx(0.01) and rep.substeps >= 1 and rep.state_revision == 1
    assert sampled.shape == (2, 2) and np.isfinite(sampled).all()
    assert state.velocity.shape == (1, sc.domain.ny, sc.domain.nx, 2)
    solid = NacaFoil(sc.foil).mask(sc.domain, state.angle_degrees)
    np.testing.assert_array_equal(state.velocity[0][solid], 0.0)
    assert all(np.isfinite(v) for v in diag.values.values()) and diag.state_revision == 1


def test_import_rejects_nonfinite_velocity_without_mutation():
    sc = _scenario()
    src, dst = _started(sc), _started(sc)
    state = src.export_state()
    state.velocity[0, 0, 0, 0] = np.nan
    before = dst.export_state()
    out = dst.import_state(state, ControlState(state.time, state.angle_degrees, state.angular_velocity_degrees))
    assert out.status == "rejected" and out.reason == "nonfinite_state"
    assert dst.state_revision == 0
    _same_state(dst.export_state(), before)


def test_import_rejects_velocity_inside_the_solid():
    sc = _scenario(64, 32)
    src, dst = _started(sc), _started(sc)
    state = src.export_state()
    solid = NacaFoil(sc.foil).mask(sc.domain, state.angle_degrees)
    vel = state.velocity.copy()
    r, c = np.argwhere(solid)[0]
    vel[0, r, c, 0] = 0.125
    before = dst.export_state()
    out = dst.import_state(replace(state, velocity=vel),
                           ControlState(state.time, state.angle_degrees, state.angular_velocity_degrees))
    assert out.status == "rejected" and out.reason == "postcondition_failure" and out.stage == "canonical-import"
    assert int(out.evidence["nonzero_solid_cells"]) > 0
    assert dst.state_revision == 0
    _same_state(dst.export_state(), before)


def test_import_whose_projection_fails_on_the_device_leaves_the_state():
    """A finite field too fast for the import projection fails inside the library; the device
    state and the revision stay as they were."""
    sc = _scenario(64, 32)
    dst = _started(sc)
    dst.advance(sc.control_at(sc.output_dt), sc.output_dt)
    before, rev = dst.export_state(), dst.state_revision
    fast = before.velocity.copy()
    solid = NacaFoil(sc.foil).mask(sc.domain, before.angle_degrees)
    fast[0][~solid] = 1.0e7
    out = dst.import_state(replace(before, velocity=fast),
                           ControlState(before.time, before.angle_degrees, before.angular_velocity_degrees))
    assert out.status == "rejected" and out.reason == "excessive_velocity"
    assert dst.state_revision == rev
    _same_state(dst.export_state(), before)


def test_postcondition_failure_rolls_back_atomically():
    sc = workloads.single("stall", 32, 16, "2412", 25.0, 1000.0, tolerance=1e-3, transport="maccormack",
                          extra={"mac_maximum_divergence_linf": 0.0, "mac_maximum_solid_leakage": 0.0,
                                 "stable_cfl": 1.25})
    s = _started(sc)
    before = s.export_state()
    with pytest.raises(NumericalFailure) as err:
        s.advance(ControlState(sc.output_dt, 25.0, 0.0), sc.output_dt)
    assert err.value.reason == "postcondition_failure" and err.value.stage == "postcondition"
    assert float(err.value.evidence["divergence_linf"]) > 0.0
    assert s.state_revision == 0
    _same_state(s.export_state(), before)


def test_invalid_limit_is_rejected_before_mutation():
    sc = _scenario()
    s = _started(sc)
    before, diag = s.export_state(), s.diagnostics()
    sc.solver_options["mac_maximum_divergence_linf"] = "invalid"
    with pytest.raises(TypeError, match="mac_maximum_divergence_linf"):
        s.advance(ControlState(sc.output_dt, before.angle_degrees, 0.0), sc.output_dt)
    assert s.state_revision == 0
    _same_state(s.export_state(), before)
    assert s.diagnostics() == diag


def test_pressure_iteration_budget_is_honoured():
    sc = _scenario(64, 32, pressure_max_iterations=1, pressure_tolerance=1e-12)
    with pytest.raises(NumericalFailure) as err:
        _started(sc)
    assert err.value.reason == "projection_failure" and err.value.stage == "projection"
    assert err.value.evidence["iterations"] == 1


def test_fresh_restart_keeps_the_declared_initial_condition():
    sc = Scenario(1, "tg", DomainSpec(2, ((0.0, 2 * np.pi), (0.0, 2 * np.pi)), (32, 32), ("x", "y")), 100.0,
                  (0.0, 0.0), FoilSpec("0012", 0.2, (-10.0, -10.0)), (ControlKeyframe(0.0, 0.0),), 1.0, 0.02,
                  "float64", 0, {"initial_condition": "taylor-green"})
    s = StableFluidsSolver()
    s.restart(sc, NacaFoil(sc.foil), sc.seed, RestartState(0.5, 0.0, sc.reynolds))
    assert float(np.max(np.abs(s.export_state().velocity[0, :, :, 1]))) > 0.25


def test_runtime_reynolds_change():
    sc = _scenario()
    s = _started(sc)
    s.set_reynolds(2.0 * sc.reynolds)
    s.advance(sc.control_at(sc.output_dt), sc.output_dt)
    assert s.reynolds == 2.0 * sc.reynolds
    assert s.diagnostics().values["requested_reynolds"] == 2.0 * sc.reynolds
    assert np.isfinite(s.export_state().velocity).all()
    with pytest.raises(ValueError, match="Reynolds"):
        s.set_reynolds(0.0)


@pytest.mark.parametrize("precision", ["float32", "float64"])
def test_deterministic_for_a_fixed_seed(precision):
    """Fixed-order reductions: two runs give bit-identical fields."""
    sc = _scenario(96, 48, precision=precision)
    a, b = _started(sc), _started(sc)
    for k in range(3):
        a.advance(sc.control_at((k + 1) * sc.output_dt), sc.output_dt)
        b.advance(sc.control_at((k + 1) * sc.output_dt), sc.output_dt)
    np.testing.assert_array_equal(a.export_state().velocity, b.export_state().velocity)
    np.testing.assert_array_equal(a.pressure(), b.pressure())


def test_import_rebuilds_faces_and_reprojects_like_the_reference():
    """Import (stable_fluids.py:636-706): solids take the wall velocity, faces are averaged from
    the cells, then a projection with a 1e-4 pseudo-step. Checked against the oracle's
    restatement of those steps, in FP64 (1e-10 absolute)."""
    from oracle.stable_fluids import OracleSolver, cell_to_faces

    sc = _scenario(64, 32, precision="float64")
    a = _started(sc)
    for k in range(2):
        a.advance(sc.control_at((k + 1) * sc.output_dt), sc.output_dt)
    st = a.export_state()
    b = _started(sc)
    ctl = ControlState(st.time, st.angle_degrees, st.angular_velocity_degrees)
    out = b.import_state(st, ctl)
    assert out.accepted and b.state_revision == 1
    o = OracleSolver(sc)
    o.initialize()
    vel = np.asarray(st.velocity[0], dtype=np.float64).copy()
    o.angle, o.omega, o.time = ctl.angle_degrees, ctl.angular_velocity_degrees, st.time
    o.solid = o._mask(ctl.angle_degrees)
    wall = o._wall(ctl.angular_velocity_degrees)
    vel[o.solid] = wall[o.solid]
    o.u, o.v = cell_to_faces(vel)
    o._project(1.0e-4)
    np.testing.assert_allclose(b.export_state().velocity[0], o.export_velocity(), rtol=0, atol=1e-10)


def test_export_uses_reusable_page_locked_blocks():
    """export_state returns an ordinary writable array backed by a page-locked block of the
    library's host pool; a freed block is handed out again for the next request of the same
    size; exported values equal the faces' cell average."""
    import ctypes

    from foilbench_b200 import _native as N

    lib = N.lib()
    size = 123 * 4096 + 48  # a size no export of these tests has
    p1, p2 = ctypes.c_void_p(), ctypes.c_void_p()
    rc = lib.fb_host_alloc(size, ctypes.byref(p1))
    assert rc == N.FB_OK, lib.fb_last_error().decode()
    assert lib.fb_host_free(p1) == N.FB_OK
    assert lib.fb_host_alloc(size, ctypes.byref(p2)) == N.FB_OK
    assert p2.value == p1.value  # the most recently freed block of the size, reused
    assert lib.fb_host_free(p2) == N.FB_OK
    assert lib.fb_host_free(ctypes.c_void_p(p2.value + 16)) != N.FB_OK  # not a pool block

    sc = _scenario(64, 32)
    s = _started(sc)
    a = s.export_state().velocity
    assert a.flags["WRITEABLE"] and a.dtype == np.float32 and a.shape == (1, 32, 64, 2)
    base = a
    while base is not None and not hasattr(base, "_block"):
        base = getattr(base, "base", None)
    assert base is not None, "export is not backed by a pool block"
    u, v = s.face_velocities()
    cell = np.stack([0.5 * (u[:, :-1] + u[:, 1:]), 0.5 * (v[:-1, :] + v[1:, :])], axis=-1)
    cell[s.solid_mask()] = 0.0
    np.testing.assert_allclose(a[0], cell, rtol=0, atol=1e-6)
    a[...] = -1.0  # the caller owns its array; the next export is unaffected
    np.testing.assert_allclose(s.export_state().velocity[0], cell, rtol=0, atol=1e-6)


def _extras():
    import json

    from tests._golden import GOLDEN

    d = np.load(GOLDEN / "extras.npz")
    return d, json.loads(str(d["meta"]))


@pytest.mark.parametrize("precision", ["float64", "float32"])
def test_sample_velocity_matches_the_reference(precision):
    """sample_velocity (stable_fluids.py:609-611): bilinear samples of the cell velocity with
    clamped edges, at points outside the domain, inside the foil and on cell centres. Two
    checks: against the oracle's restatement of sample_vector on this solver's own cell
    velocity (1e-12 in float64, float32 rounding in float32), and end to end against the
    reference's samples after three advances (1e-9 in float64; float32 fields follow the
    reference's float32 arithmetic to 2e-5 relative)."""
    from oracle.stable_fluids import Grid, sample_vector
    from foilbench_b200.models import scenario_from_dict

    d, meta = _extras()
    sc = scenario_from_dict(meta[f"sample_{precision}"])
    sc = replace(sc, solver_options={**sc.solver_options, "pressure_scheme": "reference"})
    s = _started(sc)
    for k in range(3):
        s.advance(sc.control_at((k + 1) * sc.output_dt), sc.output_dt)
    pts = d[f"sample_{precision}_points"]
    got = s.sample_velocity(pts)
    assert got.dtype == np.dtype(precision) and got.shape == (pts.shape[0], 2)
    own = sample_vector(s.cell_velocity(), pts, Grid.from_domain(sc.domain))
    np.testing.assert_allclose(got, own, rtol=0, atol=1e-12 if precision == "float64" else 1e-6)
    ref = d[f"sample_{precision}_values"]
    err = float(np.linalg.norm(got.astype(np.float64) - ref) / np.linalg.norm(ref))
    assert err < (1e-9 if precision == "float64" else 2e-5), err


def test_restart_matches_the_reference():
    """restart (stable_fluids.py:218-236): initialise, take the restart time, pose and Reynolds
    number, rebuild the mask at the restart angle, write the wall velocity (zero angular
    velocity) into the solid cells, average to faces and re-project; then advance toward a
    pitching control. Against the reference in FP64: mask bit-exact, faces and pressure 1e-9,
    equal CG iteration counts."""
    from foilbench_b200.models import scenario_from_dict

    d, meta = _extras()
    m = meta["restart"]
    sc = scenario_from_dict(m["scenario"])
    t0, angle, re = m["start"]
    s = StableFluidsSolver()
    s.restart(sc, NacaFoil(sc.foil), 0, RestartState(t0, angle, re))
    assert s.reynolds == re and s.state_revision == 0
    np.testing.assert_array_equal(s.solid_mask(), d["restart_solid0"])
    u, v = s.face_velocities()
    for got, ref in ((u, d["restart_u0"]), (v, d["restart_v0"]), (s.pressure(), d["restart_p0"])):
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-9
    assert s._last_projection["iterations"] == m["evidence"][0]
    for k in range(2):
        c = sc.control_at(t0 + (k + 1) * sc.output_dt)
        rep = s.advance(ControlState(c.time, c.angle_degrees, c.angular_velocity_degrees), sc.output_dt)
        ev = m["evidence"][k + 1]
        assert rep.substeps == ev["substeps"]
        assert rep.evidence["pressure_total_iterations"] == sum(ev["pressure_iterations"])
        u, v = s.face_velocities()
        assert np.linalg.norm(u - d[f"restart_u{k + 1}"]) / np.linalg.norm(d[f"restart_u{k + 1}"]) < 1e-9
        assert np.linalg.norm(v - d[f"restart_v{k + 1}"]) / np.linalg.norm(d[f"restart_v{k + 1}"]) < 1e-9


@pytest.mark.parametrize("precision,row_transform,barrier", [("float64", None, 1), ("float32", None, 1),
                                                             ("float32", "tensor", 30)])
def test_barrier_wait_runs_out_and_rolls_back(precision, row_transform, barrier):
    """Failure detection without a device fault: with the test hook, CTA 0 does not arrive at
    a grid barrier of the launch (the first; or, with the tensor-core row transform, one inside
    the CG loop, after tensor-core phases ran), every CTA's bounded wait runs out after 20 ms,
    the kernel returns and the advance reports FB_ERR_DEVICE_TIMEOUT with state and revision
    unchanged. With the hook off the same solver advances exactly like an untouched twin."""
    import ctypes  # noqa: F401

    from foilbench_b200 import _native as N

    if row_transform:
        sc = _scenario(96, 48, precision=precision, pressure_scheme="mixed", pressure_row_transform=row_transform)
    else:
        sc = _scenario(96, 48, precision=precision)
    a, b = _started(sc), _started(sc)
    a.advance(sc.control_at(sc.output_dt), sc.output_dt)
    b.advance(sc.control_at(sc.output_dt), sc.output_dt)
    before = a.export_state()
    assert N.lib().fb_debug_barrier_timeout(a._native.handle, barrier, 20_000_000) == N.FB_OK
    c = sc.control_at(2 * sc.output_dt)
    with pytest.raises(N.NativeError) as err:
        a.advance(c, sc.output_dt)
    assert err.value.code == N.FB_ERR_DEVICE_TIMEOUT
    assert a.state_revision == 1
    _same_state(a.export_state(), before)
    assert N.lib().fb_debug_barrier_timeout(a._native.handle, 0, 0) == N.FB_OK
    ra = a.advance(c, sc.output_dt)
    rb = b.advance(c, sc.output_dt)
    assert ra.substeps == rb.substeps and a.state_revision == 2
    np.testing.assert_array_equal(a.export_state().velocity, b.export_state().velocity)


def test_autotune_keeps_state_and_is_adopted_by_later_solvers():
    """fb_autotune times candidate launch shapes and sweep schedules on one substep of the
    solver's own state and restores that state after every trial; the winner is applied and
    cached, so solvers of the same grid created afterwards start with the same configuration,
    and two of them produce bit-identical fields."""
    sc = _scenario(256, 128, precision="float32", pressure_scheme="mixed")
    a = _started(sc)
    before = a.export_state()
    t = a.autotune(sc.output_dt, reps=2)
    assert t["trials"] >= 2 and t["tuned_ms"] > 0.0 and t["heuristic_ms"] > 0.0
    assert t["tuned_ms"] <= t["heuristic_ms"] * 1.0001
    assert t["column_tile"] in (2, 4, 8, 16) and 1 <= t["ctas"] <= t["heuristic_ctas"]
    assert a.state_revision == 0
    _same_state(a.export_state(), before)
    shape = a.launch_shape()
    assert shape["ctas"] == t["ctas"] and shape["column_tile"] == t["column_tile"]
    assert shape["inner_rtol"] == pytest.approx(t["inner_rtol"])
    c, d = _started(sc), _started(sc)
    assert c.launch_shape() == shape and d.launch_shape() == shape
    for k in range(2):
        c.advance(sc.control_at((k + 1) * sc.output_dt), sc.output_dt)
        d.advance(sc.control_at((k + 1) * sc.output_dt), sc.output_dt)
    np.testing.assert_array_equal(c.export_state().velocity, d.export_state().velocity)
    # a shape set by hand is validated and applied
    c.set_launch_shape(ctas=max(1, shape["ctas"] // 2), column_tile=4)
    assert c.launch_shape()["ctas"] == max(1, shape["ctas"] // 2) and c.launch_shape()["column_tile"] == 4
    with pytest.raises(Exception):
        c.set_launch_shape(ctas=100000)
