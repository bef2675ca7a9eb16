"""Parity of the CUDA path with the reference: geometry, single operators and multi-step
solver trajectories, through the C ABI (foilbench_b200 -> libfoilb200.so).

Tolerances (written per assertion):
* masks: bit-exact; signed distance 1e-13 absolute.
* FP64 operators: 1e-12 (advection, viscosity), 1e-10 relative pressure; equal CG and
  Jacobi iteration counts.
* FP64 trajectories (reference pressure scheme): 1e-9 relative L2 on u, v, equal
  substep / CG / Jacobi counts.
* float32 fields with the reference (FP64) pressure scheme: 2e-5 relative L2.
* float32 fields with the mixed scheme against the reference's own float32 trajectories:
  5e-5 relative L2 (the two differ in arithmetic: the reference evaluates its stencils in
  float32, the mixed scheme in FP64). Against the FP64 reference the mixed scheme is held to
  1e-5 (tests/test_gpu_precision.py).
* passive scalar and the fixed sweep count: against the oracle, tolerances in each test.
"""

from dataclasses import replace

import numpy as np
import pytest

from foilbench_b200.geometry import NacaFoil
from foilbench_b200.models import ControlState, DomainSpec, FoilSpec
from foilbench_b200.solver import StableFluidsSolver
from foilbench_b200 import grid_ops as G
from tests._golden import TRAJECTORIES, Trajectory, geometry, masks, operators

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_device_masks_match_reference_bit_for_bit():
    for meta, ref in masks():
        dom = DomainSpec(2, tuple(tuple(b) for b in meta["bounds"]), tuple(meta["resolution"]))
        foil = NacaFoil(FoilSpec(meta["naca"], meta["chord"], tuple(meta["pivot"])))
        got = foil.mask(dom, meta["angle_degrees"])
        assert int(got.sum()) == meta["solid_cells"], meta["name"]
        np.testing.assert_array_equal(got, ref)


def test_device_signed_distance_matches_reference():
    for rec in geometry():
        f = rec["foil"]
        foil = NacaFoil(FoilSpec(f["naca"], f["chord"], tuple(f["pivot"])))
        for q in rec["queries"]:
            pts = np.asarray(q["points"], dtype=np.float64)
            d = foil.signed_distance(pts, q["angle_degrees"])
            np.testing.assert_allclose(d, q["signed_distance"], rtol=0, atol=1e-13)
            np.testing.assert_array_equal(d <= 0.0, np.asarray(q["contains"]))
            np.testing.assert_allclose(foil.normals(pts, q["angle_degrees"]), q["normals"], rtol=0, atol=1e-8)


def _dom(meta):
    return DomainSpec(2, tuple(tuple(b) for b in meta["bounds"]), tuple(meta["resolution"]),
                      tuple(meta.get("periodic_axes", ())))


@pytest.mark.parametrize("tag", ["clamp", "periodic"])
def test_advection_matches_reference(tag):
    d, meta = operators()
    m = meta[f"adv_{tag}"]
    dom = _dom(m)
    vel = d[f"adv_{tag}_in"]
    np.testing.assert_allclose(G.advect_velocity(vel, m["dt"], dom, False), d[f"adv_{tag}_sl"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(G.advect_velocity(vel, m["dt"], dom, True), d[f"adv_{tag}_mc"], rtol=0, atol=1e-12)
    got32 = G.advect_velocity(d[f"adv_{tag}_in32"], m["dt"], dom, True)
    assert got32.dtype == np.float32
    np.testing.assert_allclose(got32, d[f"adv_{tag}_mc32"], rtol=0, atol=2e-6)


@pytest.mark.parametrize("tag", ["clamp", "periodic"])
def test_viscosity_matches_reference(tag):
    d, meta = operators()
    m = meta[f"dif_{tag}"]
    dom = _dom(meta[f"adv_{tag}"])
    out, rep = G.implicit_diffuse(d[f"adv_{tag}_in"], m["nu"], m["dt"], dom, m["tol"], 640)
    assert rep.converged and rep.iterations == m["iterations"]
    np.testing.assert_allclose(out, d[f"dif_{tag}_out"], rtol=0, atol=1e-12)


def test_periodic_face_viscosity_known_answer():
    # discrete Fourier decay 1/(1 + nu dt 4 sin^2(pi/n)/dx^2) (reference test_projection.py:90)
    dom = DomainSpec(2, ((0.0, 2.0), (0.0, 1.0)), (32, 16), ("x", "y"))
    phase = 2.0 * np.pi * np.arange(dom.nx) / dom.nx
    vel = np.zeros((dom.ny, dom.nx, 2))
    vel[:, :, 0] = np.sin(phase)[None, :]
    nu, dt = 0.2, 0.03
    out, rep = G.implicit_diffuse(vel, nu, dt, dom, 1.0e-10)
    factor = 1.0 / (1.0 + nu * dt * 4.0 * np.sin(np.pi / dom.nx) ** 2 / dom.dx**2)
    assert rep.converged
    np.testing.assert_allclose(out[:, :, 0], factor * vel[:, :, 0], atol=1e-8)


@pytest.mark.parametrize("tag", ["dst", "dst_odd", "jac_x", "jac_xy"])
def test_masked_poisson_matches_reference(tag):
    d, meta = operators()
    m = meta[f"poi_{tag}"]
    p, info, iters, rel = G.solve_masked_poisson(d[f"poi_{tag}_rhs"], d[f"poi_{tag}_fluid"], m["dx"], m["dy"],
                                                 tuple(m["periodic_axes"]), m["tol"], 640)
    assert info == 0
    assert iters == m["iterations"]
    assert rel == pytest.approx(m["relative_residual"], rel=1e-4)
    assert _rel(p, d[f"poi_{tag}_p"]) < 1e-10


@pytest.mark.parametrize("tag", ["dst", "dst_odd", "jac_x", "jac_xy"])
def test_mixed_poisson_meets_tolerance(tag):
    d, meta = operators()
    m = meta[f"poi_{tag}"]
    p, info, iters, rel = G.solve_masked_poisson(d[f"poi_{tag}_rhs"], d[f"poi_{tag}_fluid"], m["dx"], m["dy"],
                                                 tuple(m["periodic_axes"]), m["tol"], 640, scheme="mixed")
    assert info == 0 and rel <= m["tol"] * (1 + 1e-6)
    assert _rel(p, d[f"poi_{tag}_p"]) < 50 * m["tol"]


def test_face_projection_matches_reference():
    d, meta = operators()
    m = meta["prj"]
    dom = DomainSpec(2, ((-2.0, 2.0), (-1.0, 1.0)), (64, 32))
    u, v, rep = G.project_faces(d["prj_u_in"], d["prj_v_in"], dom, d["prj_solid"], 0.0, (1.0, 0.0), m["dt"],
                                pressure_tolerance=m["tol"])
    assert rep.converged and rep.iterations == m["iterations"]
    np.testing.assert_allclose(u, d["prj_u_out"], rtol=0, atol=1e-11)
    np.testing.assert_allclose(v, d["prj_v_out"], rtol=0, atol=1e-11)


def _run(t: Trajectory, scheme: str | None = None):
    sc = t.scenario
    if scheme is not None:
        sc = replace(sc, solver_options={**sc.solver_options, "pressure_scheme": scheme})
    s = StableFluidsSolver()
    s.initialize(sc, NacaFoil(sc.foil), 0)
    return sc, s


@pytest.mark.parametrize("name", TRAJECTORIES)
def test_trajectory_matches_reference(name):
    t = Trajectory(name)
    fp32 = t.scenario.precision == "float32"
    # The Poiseuille start is exactly divergence-free, so every projection solves a system
    # whose right-hand side is rounding noise; CG iteration counts on noise are not
    # reproducible between implementations (fields still agree to the stated tolerance).
    noise_rhs = name.startswith("poiseuille")
    sc, s = _run(t, "reference")
    tol = 2e-5 if fp32 else 1e-9
    u0, v0 = s.face_velocities()
    np.testing.assert_array_equal(s.solid_mask(), t["solid0"])
    assert _rel(u0, t["u0"]) < tol and _rel(v0, t["v0"]) < 10 * tol
    for k in range(t.steps):
        ev = t.evidence[k + 1]
        c = sc.control_at((k + 1) * t.dt)
        rep = s.advance(ControlState(c.time, c.angle_degrees, c.angular_velocity_degrees), t.dt)
        assert rep.substeps == ev["substeps"], (k, rep.substeps, ev["substeps"])
        if not fp32 and not noise_rhs:
            assert rep.evidence["pressure_iterations"] == ev["pressure_iterations"], k
            assert rep.evidence["viscosity_iterations"] == ev["viscosity_iterations"], k
        if t.has(f"u{k + 1}"):
            u, v = s.face_velocities()
            assert _rel(u, t[f"u{k + 1}"]) < tol, (k, _rel(u, t[f"u{k + 1}"]))
            # v relative to the whole velocity scale: in channel flow v is rounding noise
            vscale = np.linalg.norm(t[f"v{k + 1}"]) + np.linalg.norm(t[f"u{k + 1}"])
            assert np.linalg.norm(v - t[f"v{k + 1}"]) / vscale < 10 * tol
            if not noise_rhs:
                assert _rel(s.pressure(), t[f"p{k + 1}"]) < (1e-3 if fp32 else 1e-7)
    np.testing.assert_array_equal(s.solid_mask(), t["solid_final"])
    assert _rel(s.export_state().velocity[0], t["export"]) < tol
    diag = s.diagnostics().values
    for key in ("kinetic_energy", "enstrophy", "divergence_l2", "wake_width", "recirculation_area"):
        assert diag[key] == pytest.approx(t.diagnostics[key], rel=1e-4 if fp32 else 1e-7, abs=1e-9), key


@pytest.mark.parametrize("name", [n for n in TRAJECTORIES if "float32" in n or "helper" in n or "stall" in n])
def test_mixed_scheme_trajectory_tracks_reference(name):
    t = Trajectory(name)
    sc, s = _run(t, "mixed")
    for k in range(t.steps):
        c = sc.control_at((k + 1) * t.dt)
        rep = s.advance(ControlState(c.time, c.angle_degrees, c.angular_velocity_degrees), t.dt)
        assert rep.evidence["pressure_relative_residual"] <= sc.solver_options.get("pressure_tolerance", 1e-5) * (1 + 1e-6)
        if t.has(f"u{k + 1}"):
            u, _ = s.face_velocities()
            assert _rel(u, t[f"u{k + 1}"]) < 5e-5, (k, _rel(u, t[f"u{k + 1}"]))


@pytest.mark.parametrize("nx,ny,scheme,rt", [(200, 24, "reference", "fft"), (1040, 24, "reference", "fft"),
                                             (2064, 24, "reference", "fft"), (2064, 24, "mixed", "fft"),
                                             (4112, 24, "mixed", "fft"), (2064, 24, "mixed", "tensor"),
                                             (4112, 24, "mixed", "tensor"), (770, 200, "mixed", "tensor"),
                                             (61, 131, "mixed", "tensor"), (8192, 24, "reference", "fft"),
                                             (5001, 20, "reference", "fft")])
def test_masked_poisson_every_transform_shape(nx, ny, scheme, rt):
    """Row-transform shapes: 512-point (three passes), 4096-point FP64 and 8192/16384-point
    FP32 (four passes, long rows) and 8192-point FP64 (run-time plan), FP64 rows over 4096
    points as two half convolutions (8192 x 24: equal halves; 5001 x 20: odd length, ragged
    second half), and the tensor-core
    transform on whole, ragged (770 x 200: partial tiles of rows, wavenumbers and sum
    indices) and odd (61 x 131: a self-mirrored wavenumber, unaligned rows) grids, against the
    oracle's restatement of the reference solve on the same seeded right-hand side. The FP64
    scheme takes the oracle's iterations to 1e-10; the mixed scheme meets the tolerance within
    50 x tol of the oracle's pressure."""
    from oracle.stable_fluids import solve_masked_poisson as oracle_solve

    tol = 1e-8
    rng = np.random.default_rng(nx)
    fluid = np.ones((ny, nx), dtype=bool)
    fluid[8:15, nx // 3:nx // 3 + max(1, nx // 20)] = False
    rhs = np.where(fluid, rng.normal(size=(ny, nx)), 0.0)
    dx, dy = 4.0 / nx, 2.0 / ny
    p_ref, info_ref, it_ref, rel_ref = oracle_solve(rhs, fluid, dx, dy, (), tol, 640)
    p, info, iters, rel = G.solve_masked_poisson(rhs, fluid, dx, dy, (), tol, 640, scheme=scheme, row_transform=rt)
    assert info == 0 and info_ref == 0
    if scheme == "reference":
        assert iters == it_ref
        assert _rel(p, p_ref) < 1e-10
    else:
        assert rel <= tol * (1 + 1e-6)
        assert _rel(p, p_ref) < 50 * tol


@pytest.mark.parametrize("nx,ny,periodic,scheme", [
    (4, 12, (), "reference"),            # one lane owns both strip edges
    (8, 10, ("x",), "reference"),        # two lanes, periodic wrap through the edge loads
    (132, 20, (), "reference"),          # second strip of one lane
    (136, 18, ("x",), "reference"),      # second strip of two lanes, periodic x
    (260, 22, ("y",), "reference"),      # third strip of one lane, periodic y (Jacobi)
    (200, 16, ("x", "y"), "reference"),  # doubly periodic (singular, mean removed)
    (130, 14, (), "reference"),          # width not a multiple of 4: the per-cell path
    (392, 40, (), "mixed"),              # float32 Krylov vectors, partial last strip
])
def test_masked_poisson_operator_strip_edges(nx, ny, periodic, scheme):
    """The CG direction/operator phase walks 128-column strips with four cells per lane; strip
    edges, partial strips, one-lane strips and periodic wraps all go through the masked
    operator, checked against the oracle's restatement of the reference solve (same
    iteration count in float64)."""
    from oracle.stable_fluids import solve_masked_poisson as oracle_solve

    tol = 1e-8
    rng = np.random.default_rng(nx * 1000 + ny)
    # solid blocks across the strip boundaries (columns 127 | 128) and at the last columns
    fluid = np.ones((ny, nx), dtype=bool)
    fluid[ny // 4:ny // 2, max(0, min(nx, 128) - 3):min(nx, 131)] = False
    fluid[ny // 2 + 1:ny - 2, nx - 2:nx] = False
    rhs = np.where(fluid, rng.normal(size=(ny, nx)), 0.0)
    dx, dy = 1.0 / nx, 1.3 / ny
    p_ref, info_ref, it_ref, _ = oracle_solve(rhs, fluid, dx, dy, periodic, tol, 2000)
    p, info, iters, rel = G.solve_masked_poisson(rhs, fluid, dx, dy, periodic, tol, 2000, scheme=scheme)
    assert info == 0 and info_ref == 0
    if len(periodic) == 2:  # singular: compare up to the constant
        p = p - p[fluid].mean()
        p_ref = p_ref - p_ref[fluid].mean()
    if scheme == "reference":
        # DST-preconditioned solves take the oracle's iteration count; the periodic
        # (Jacobi-preconditioned) runs take hundreds of iterations and may stop one apart,
        # their dot products being summed in another order
        assert abs(iters - it_ref) <= (1 if periodic else 0), (iters, it_ref)
        assert _rel(p, p_ref) < 1e-9
    else:
        assert rel <= tol * (1 + 1e-6)
        assert _rel(p, p_ref) < 100 * tol


@pytest.mark.parametrize("scheme,tol", [("reference", 1e-10), ("mixed", 1e-4)])
def test_fixed_sweep_count_matches_the_oracle(scheme, tol):
    """The sweep rule of the bandwidth stress configuration (pressure_fixed_iterations): exactly
    N PCG iterations per projection, no early exit, even where the tolerance would stop the
    iteration sooner. Against the oracle's restatement of the reference solve run with the same
    N and a zero tolerance (scipy's loop then runs all N iterations). FP64: 1e-10 relative; the
    mixed scheme runs the N sweeps in FP32 and corrects once in FP64, 1e-4 relative."""
    from oracle.stable_fluids import solve_masked_poisson as oracle_solve

    ny, nx, n = 64, 128, 8
    rng = np.random.default_rng(77)
    fluid = np.ones((ny, nx), dtype=bool)
    fluid[20:34, 40:52] = False
    rhs = np.where(fluid, rng.normal(size=(ny, nx)), 0.0)
    dx, dy = 4.0 / nx, 2.0 / ny
    p_ref, info_ref, it_ref, rel_ref = oracle_solve(rhs, fluid, dx, dy, (), 0.0, n)
    assert it_ref == n and info_ref == n
    # the tolerance alone would stop after fewer iterations
    _, _, it_free, _ = G.solve_masked_poisson(rhs, fluid, dx, dy, (), 1e-2, 640, scheme=scheme)
    assert it_free < n
    p, info, iters, rel = G.solve_masked_poisson(rhs, fluid, dx, dy, (), 1e-2, 640, scheme=scheme,
                                                 fixed_iterations=n)
    assert info == 0 and iters == n
    assert _rel(p, p_ref) < tol, _rel(p, p_ref)
    if scheme == "reference":
        assert rel == pytest.approx(rel_ref, rel=1e-6)
    else:  # the FP32 sweeps' own rounding sits near 1e-7 of the right-hand side
        assert rel < 2.0 * rel_ref + 1e-6


@pytest.mark.parametrize("precision,scheme,tol", [("float64", "reference", 1e-11), ("float32", "mixed", 1e-5)])
def test_passive_scalar_matches_the_oracle(precision, scheme, tol):
    """Passive scalar (no reference counterpart; carried by the bandwidth stress configuration):
    each substep samples the scalar at the departure point of the velocity's own RK2 trace,
    as oracle.advect_scalar composes rk2_backtrace (PY/core/grid.py:527) with sample_scalar
    (PY/core/interpolation.py:55). Against the oracle in FP64 over four advances: 1e-11
    relative in FP64, 1e-5 for float32 fields with the mixed scheme."""
    from foilbench_b200 import workloads
    from oracle.stable_fluids import OracleSolver, cell_centers

    sc = workloads.single("scalar", 64, 32, "2412", 10.0, 800.0, precision=precision, tolerance=1e-9,
                          scheme=scheme, extra={"passive_scalar": True})
    s = StableFluidsSolver()
    s.initialize(sc, NacaFoil(sc.foil), 0)
    sc64 = replace(sc, precision="float64", solver_options={**sc.solver_options, "pressure_scheme": "reference"})
    o = OracleSolver(sc64)
    o.initialize()
    pos = cell_centers(o.grid)
    rng = np.random.default_rng(3)
    c0 = np.exp(-((pos[:, :, 0] - 0.6) ** 2 + pos[:, :, 1] ** 2) / 0.08) + 0.05 * rng.normal(size=pos.shape[:2])
    s.set_passive_scalar(c0)
    o.scalar = np.asarray(c0, dtype=np.dtype(precision)).astype(np.float64)
    for k in range(4):
        c = sc.control_at((k + 1) * sc.output_dt)
        rep = s.advance(ControlState(c.time, c.angle_degrees, c.angular_velocity_degrees), sc.output_dt)
        orc = o.advance(c, sc.output_dt)
        assert rep.substeps == orc.substeps
    got = s.passive_scalar()
    assert got.dtype == np.dtype(precision)
    assert _rel(got, o.scalar) < tol, _rel(got, o.scalar)
    assert _rel(got, c0) > 1e-3  # the scalar moved


def test_fp64_rows_over_4096_points_advance_like_the_oracle():
    """A whole FP64 advance on a grid whose rows exceed one shared-memory convolution (4160
    columns: the preconditioner's row DST runs as two half convolutions) against the oracle's
    restatement of the reference advance (PY/solvers/stable_fluids.py:332-603): equal substep
    and pressure iteration counts, velocity to 1e-9 over three advances."""
    from foilbench_b200 import workloads
    from oracle.stable_fluids import OracleSolver

    sc = workloads.single("wide", 4160, 24, "0012", 6.0, 500.0, precision="float64", tolerance=1e-8)
    s = StableFluidsSolver()
    s.initialize(sc, NacaFoil(sc.foil), 0)
    o = OracleSolver(sc)
    o.initialize()
    for k in range(3):
        c = sc.control_at((k + 1) * sc.output_dt)
        rep = s.advance(ControlState(c.time, c.angle_degrees, c.angular_velocity_degrees), sc.output_dt)
        orc = o.advance(c, sc.output_dt)
        assert rep.substeps == orc.substeps
        assert rep.evidence["pressure_iterations"] == orc.evidence["pressure_iterations"]
    assert _rel(s.export_state().velocity[0], o.export_velocity()) < 1e-9
