"""Pin the CPU oracle against fixtures produced by running the reference itself.

Tolerances: geometry and single operators agree to rounding (1e-12 .. 1e-14);
multi-step FP64 trajectories to 1e-9 relative with identical CG/Jacobi iteration
counts and substep counts; FP32 trajectories to 1e-5 (float32 storage).
"""

import json

import numpy as np
import pytest

from oracle import stable_fluids as O
from foilbench_b200.models import ControlState
from tests._golden import TRAJECTORIES, Trajectory, geometry, masks, operators


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_geometry_matches_reference_and_published_vectors():
    for rec in geometry():
        f = rec["foil"]
        up, lo = O.naca_surfaces(f["naca"], f["chord"], np.asarray(rec["surface_x"]))
        np.testing.assert_allclose(up, rec["surface_upper"], rtol=0, atol=1e-15)
        np.testing.assert_allclose(lo, rec["surface_lower"], rtol=0, atol=1e-15)
        if "published_upper" in rec:
            np.testing.assert_allclose(up, rec["published_upper"], rtol=0, atol=1e-12)
            np.testing.assert_allclose(lo, rec["published_lower"], rtol=0, atol=1e-12)
        assert O.naca_maximum_radius(f["naca"], f["chord"]) == pytest.approx(rec["maximum_radius"], abs=1e-15)
        for q in rec["queries"]:
            pts = np.asarray(q["points"], dtype=np.float64)
            d = O.naca_signed_distance(f["naca"], f["chord"], f["pivot"], pts, q["angle_degrees"])
            np.testing.assert_allclose(d, q["signed_distance"], rtol=0, atol=1e-14)
            assert ((d <= 0.0) == np.asarray(q["contains"])).all()
            if q.get("published_contains") is not None:
                assert ((d <= 0.0) == np.asarray(q["published_contains"])).all()
                np.testing.assert_allclose(d, q["published_signed_distance"], atol=1e-9)


def test_masks_match_reference_bit_for_bit():
    for meta, ref in masks():
        (x0, x1), (y0, y1) = meta["bounds"]
        g = O.Grid(meta["resolution"][0], meta["resolution"][1], x0, x1, y0, y1)
        got = O.naca_mask(meta["naca"], meta["chord"], meta["pivot"], g, meta["angle_degrees"])
        assert got.sum() == meta["solid_cells"]
        np.testing.assert_array_equal(got, ref)


def _grid(meta):
    (x0, x1), (y0, y1) = meta["bounds"]
    axes = meta.get("periodic_axes", [])
    return O.Grid(meta["resolution"][0], meta["resolution"][1], x0, x1, y0, y1, "x" in axes, "y" in axes)


def test_dst1_matches_scipy_call_site_transform():
    d, _ = operators()
    got = O.dst1_ortho(O.dst1_ortho(d["dst_in"], 0), 1)
    np.testing.assert_allclose(got, d["dst_out"], rtol=0, atol=1e-13)


@pytest.mark.parametrize("tag", ["clamp", "periodic"])
def test_advection_and_viscosity_operators(tag):
    d, meta = operators()
    g = _grid(meta[f"adv_{tag}"])
    dt = meta[f"adv_{tag}"]["dt"]
    vel = d[f"adv_{tag}_in"]
    np.testing.assert_allclose(O.advect_velocity(vel, dt, g, False), d[f"adv_{tag}_sl"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(O.advect_velocity(vel, dt, g, True), d[f"adv_{tag}_mc"], rtol=0, atol=1e-14)
    got32 = O.advect_velocity(d[f"adv_{tag}_in32"], dt, g, True)
    assert got32.dtype == np.float32
    np.testing.assert_array_equal(got32, d[f"adv_{tag}_mc32"])
    m = meta[f"dif_{tag}"]
    out, iters, resid, ok = O.implicit_diffuse(vel, m["nu"], m["dt"], g, m["tol"], 640)
    assert ok and iters == m["iterations"]
    np.testing.assert_allclose(out, d[f"dif_{tag}_out"], rtol=0, atol=1e-14)


@pytest.mark.parametrize("tag", ["dst", "dst_odd", "jac_x", "jac_xy"])
def test_masked_poisson_solves(tag):
    d, meta = operators()
    m = meta[f"poi_{tag}"]
    p, info, iters, rel = O.solve_masked_poisson(d[f"poi_{tag}_rhs"].copy(), d[f"poi_{tag}_fluid"], m["dx"], m["dy"],
                                                 tuple(m["periodic_axes"]), m["tol"], 640)
    assert info == m["info"] == 0
    assert iters == m["iterations"]
    assert rel == pytest.approx(m["relative_residual"], rel=1e-6)
    assert _rel(p, d[f"poi_{tag}_p"]) < 1e-12


def test_face_projection():
    d, meta = operators()
    m = meta["prj"]
    g = O.Grid(64, 32, -2.0, 2.0, -1.0, 1.0)
    wall = np.zeros((32, 64, 2))
    u, v, rep = O.project_faces(d["prj_u_in"].copy(), d["prj_v_in"].copy(), g, d["prj_solid"], wall, (1.0, 0.0),
                                m["dt"], False, m["tol"], 640)
    assert rep.converged and rep.iterations == m["iterations"]
    np.testing.assert_allclose(u, d["prj_u_out"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(v, d["prj_v_out"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("name", TRAJECTORIES)
def test_trajectory_matches_reference(name):
    t = Trajectory(name)
    sc = t.scenario
    solver = O.OracleSolver(sc, keep_pressure=True)
    solver.initialize()
    fp32 = sc.precision == "float32"
    tol = 2e-5 if fp32 else 1e-9
    assert t.evidence[0]["init_pressure_iterations"] == solver.last_projection.iterations
    np.testing.assert_array_equal(solver.solid, t["solid0"])
    assert _rel(solver.u, t["u0"]) < tol
    for k in range(t.steps):
        ev = t.evidence[k + 1]
        ctl = sc.control_at((k + 1) * t.dt)
        step = solver.advance(ControlState(ctl.time, ctl.angle_degrees, ctl.angular_velocity_degrees), t.dt)
        assert step.substeps == ev["substeps"], (k, step.substeps, ev["substeps"])
        if not fp32:
            assert step.evidence["pressure_iterations"] == ev["pressure_iterations"]
            assert step.evidence["viscosity_iterations"] == ev["viscosity_iterations"]
        if t.has(f"u{k + 1}"):
            assert _rel(solver.u, t[f"u{k + 1}"]) < tol
            assert _rel(solver.v, t[f"v{k + 1}"]) < tol * 10
            assert _rel(solver.pressure, t[f"p{k + 1}"]) < (1e-3 if fp32 else 1e-7)
    np.testing.assert_array_equal(solver.solid, t["solid_final"])
    assert _rel(solver.export_velocity(), t["export"]) < tol
    diag = solver.diagnostics()
    for key in ("kinetic_energy", "enstrophy", "divergence_l2", "wake_width", "recirculation_area"):
        assert diag[key] == pytest.approx(t.diagnostics[key], rel=1e-4 if fp32 else 1e-7, abs=1e-9), key


def test_surface_forces_of_uniform_pressure_vanish_and_shear_is_odd():
    """The oracle's force restatement on analytic fields: a uniform pressure exerts no net force
    on a closed body; a uniform stream of speed U over a body at rest drags it along +x."""
    import numpy as np

    from oracle.stable_fluids import Grid, naca_mask, surface_forces

    g = Grid(96, 48, -1.0, 3.0, -1.0, 1.0)
    solid = naca_mask("0012", 1.0, (0.0, 0.0), g, 5.0)
    ny, nx = solid.shape
    u = np.zeros((ny, nx + 1))
    v = np.zeros((ny + 1, nx))
    f = surface_forces(u, v, np.full((ny, nx), 3.7), solid, g, 0.01, 0.0, (0.0, 0.0), (1.0, 0.0), 1.0)
    assert abs(f["pressure_x"]) < 1e-12 and abs(f["pressure_y"]) < 1e-12
    u[:] = 1.0
    f = surface_forces(u, v, np.zeros((ny, nx)), solid, g, 0.01, 0.0, (0.0, 0.0), (1.0, 0.0), 1.0)
    assert f["viscous_x"] > 0.0 and abs(f["viscous_y"]) < 1e-12
    assert f["drag_coefficient"] == pytest.approx(2.0 * f["force_x"])
