"""Generate golden fixtures by running the reference Python Stable Fluids path.

Run from the repository root in an environment where the reference checkout is
available (it is read, never modified):

    python tests/golden/make_golden.py --reference /root/reference

The reference imports ``einx``, which is not installed here; ``_shims/einx.py``
provides the two reductions its Stable Fluids path uses. Every fixture is written
with its inputs, so tests never need the reference at run time.

Outputs (all under ``tests/golden/``):
  geometry.json        NACA surfaces / signed distance / normals / containment / wall
                       velocity, on the reference's own conformance points plus seeded
                       extra points and foils.
  masks.npz            packed solid masks for several grids, foils and angles.
  operators.npz        advection (SL, MacCormack), Jacobi viscosity, Poisson solves
                       (DST and Jacobi preconditioned, singular periodic) and face
                       projections on seeded inputs.
  traj_<name>.npz      multi-step solver trajectories: face velocities after every
                       advance (or after the listed ones), the last pressure, and the
                       per-advance evidence.
  c2full_2048x1024.npz one advance of the full-size 2048x1024 C2 scenario in FP64: the
                       evidence, row and column sums and a strided subsample of u, v and
                       the pressure after initialisation and after the advance (the full
                       fields are 50 MB; the summaries pin them at test tolerance).
  extras.npz           sample_velocity at seeded points and a restart (pose, Reynolds
                       number, wall fill, re-projection) followed by two advances.
"""

from __future__ import annotations

import argparse
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def _import_reference(root: Path):
    sys.path.insert(0, str(HERE / "_shims"))
    sys.path.insert(0, str(root / "implementations" / "python" / "src"))
    import foilbench_py.core.grid as grid_mod  # noqa: F401

    return grid_mod


def scenario_dict(sc) -> dict:
    return {
        "schema_version": sc.schema_version,
        "id": sc.id,
        "dimension": sc.domain.dimension,
        "bounds": [list(b) for b in sc.domain.bounds],
        "resolution": list(sc.domain.resolution),
        "periodic_axes": list(sc.domain.periodic_axes),
        "reynolds": sc.reynolds,
        "freestream": list(sc.freestream),
        "foil": {"naca": sc.foil.naca, "chord": sc.foil.chord, "pivot": list(sc.foil.pivot)},
        "controls": [{"time": k.time, "angle_degrees": k.angle_degrees} for k in sc.controls],
        "duration": sc.duration,
        "output_dt": sc.output_dt,
        "precision": sc.precision,
        "seed": sc.seed,
        "solver_options": dict(sc.solver_options),
    }


def make_scenario(M, *, sid, bounds, resolution, naca, angle, re, precision, options, periodic=(),
                  pivot=(0.0, 0.0), controls=None, output_dt=0.01, freestream=(1.0, 0.0), chord=1.0):
    ctrl = controls if controls is not None else [(0.0, angle)]
    return M.Scenario(
        schema_version=1,
        id=sid,
        domain=M.DomainSpec(2, tuple(tuple(b) for b in bounds), tuple(resolution), tuple(periodic)),
        reynolds=re,
        freestream=tuple(freestream),
        foil=M.FoilSpec(naca=naca, chord=chord, pivot=tuple(pivot)),
        controls=tuple(M.ControlKeyframe(t, a) for t, a in ctrl),
        duration=10.0,
        output_dt=output_dt,
        precision=precision,
        seed=0,
        solver_options=dict(options),
    )


def gen_geometry(root: Path, out: Path) -> None:
    from foilbench_py.core.geometry import NacaFoil
    from foilbench_py.core.models import ControlState, FoilSpec

    cases = []
    for name in ("naca2412.json", "geometry-v1.json"):
        doc = json.loads((root / "spec" / "conformance" / name).read_text())
        foil_doc = doc.get("foil") or doc.get("descriptor")
        cases.append({"source": f"spec/conformance/{name}", "doc": doc, "foil": foil_doc})
    rng = np.random.default_rng(2024)
    extra = []
    for naca, chord, pivot in (("0012", 1.0, (0.0, 0.0)), ("2412", 1.0, (0.1, -0.2)), ("4418", 0.7, (0.3, 0.1)),
                               ("0009", 1.3, (-0.2, 0.05))):
        pts = rng.uniform(-1.0, 2.0, (48, 2))
        pts[:, 1] *= 0.4
        extra.append({"foil": {"naca": naca, "chord": chord, "pivot": list(pivot)},
                      "points": pts.tolist(), "angles": [-5.0, 0.0, 8.0, 15.0, 25.0]})
    records = []
    for case in cases:
        f = case["foil"]
        foil = NacaFoil(FoilSpec(f["naca"], float(f["chord"]), tuple(f["pivot"])))
        doc = case["doc"]
        sx = np.asarray(doc["surface_x"], dtype=np.float64)
        up, lo = foil.surfaces(sx)
        queries = doc.get("queries") or [{"points": doc["points"], "angle_degrees": doc["angle_degrees"]}]
        qrec = []
        for q in queries:
            pts = np.asarray(q["points"], dtype=np.float64)
            ang = float(q["angle_degrees"])
            qrec.append({
                "points": pts.tolist(), "angle_degrees": ang,
                "signed_distance": foil.signed_distance(pts, ang).tolist(),
                "normals": foil.normals(pts, ang).tolist(),
                "contains": foil.contains(pts, ang).tolist(),
                "published_signed_distance": q.get("signed_distance"),
                "published_contains": q.get("contains"),
            })
        records.append({"source": case["source"], "foil": f, "surface_x": sx.tolist(),
                        "surface_upper": up.tolist(), "surface_lower": lo.tolist(),
                        "published_upper": doc["surface_upper"], "published_lower": doc["surface_lower"],
                        "maximum_radius": foil.maximum_radius, "queries": qrec})
    for case in extra:
        f = case["foil"]
        foil = NacaFoil(FoilSpec(f["naca"], float(f["chord"]), tuple(f["pivot"])))
        pts = np.asarray(case["points"])
        sx = np.linspace(-0.1, 1.1, 25) * f["chord"]
        up, lo = foil.surfaces(sx)
        qrec = []
        for ang in case["angles"]:
            qrec.append({
                "points": pts.tolist(), "angle_degrees": ang,
                "signed_distance": foil.signed_distance(pts, ang).tolist(),
                "normals": foil.normals(pts, ang).tolist(),
                "contains": foil.contains(pts, ang).tolist(),
                "wall_velocity_omega_37": foil.wall_velocity(pts, ControlState(0.0, ang, 37.0)).tolist(),
            })
        records.append({"source": "seeded", "foil": f, "surface_x": sx.tolist(), "surface_upper": up.tolist(),
                        "surface_lower": lo.tolist(), "maximum_radius": foil.maximum_radius, "queries": qrec})
    (out / "geometry.json").write_text(json.dumps({"records": records}, indent=1))


def gen_masks(out: Path) -> None:
    from foilbench_py.core.geometry import NacaFoil
    from foilbench_py.core.models import DomainSpec, FoilSpec

    cases = [
        ("c1", ((-1.0, 3.0), (-1.0, 1.0)), (256, 128), "0012", 1.0, (0.0, 0.0), 8.0),
        ("c2", ((-1.0, 3.0), (-1.0, 1.0)), (2048, 1024), "2412", 1.0, (0.0, 0.0), 15.0),
        ("helper", ((-2.0, 6.0), (-2.0, 2.0)), (48, 24), "2412", 1.0, (0.0, 0.0), 4.0),
        ("default", ((-1.5, 3.5), (-1.5, 1.5)), (160, 96), "2412", 1.0, (0.0, 0.0), 25.0),
        ("odd", ((-1.3, 2.9), (-0.9, 1.1)), (203, 97), "4415", 0.8, (0.15, -0.05), -7.5),
        ("fine", ((-0.5, 1.5), (-0.5, 0.5)), (512, 256), "0018", 1.0, (0.0, 0.0), 33.0),
    ]
    data = {}
    meta = []
    for name, bounds, res, naca, chord, pivot, ang in cases:
        dom = DomainSpec(2, bounds, res)
        m = NacaFoil(FoilSpec(naca, chord, pivot)).mask(dom, ang)
        data[name] = np.packbits(m.ravel())
        meta.append({"name": name, "bounds": [list(b) for b in bounds], "resolution": list(res), "naca": naca,
                     "chord": chord, "pivot": list(pivot), "angle_degrees": ang, "solid_cells": int(m.sum())})
    data["meta"] = np.asarray(json.dumps(meta))
    np.savez_compressed(out / "masks.npz", **data)


def gen_operators(out: Path, grid_mod) -> None:
    from foilbench_py.core._scipy_adapter import solve_masked_poisson
    from foilbench_py.core.models import DomainSpec

    rng = np.random.default_rng(11)
    data = {}
    meta = {}
    # advection on a smooth random field, clamped and periodic domains
    for tag, dom in (("clamp", DomainSpec(2, ((-1.0, 1.5), (-0.5, 0.7)), (40, 24))),
                     ("periodic", DomainSpec(2, ((0.0, 2.0), (0.0, 1.0)), (32, 16), ("x", "y")))):
        ny, nx = dom.ny, dom.nx
        yy, xx = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
        vel = np.stack((0.8 + 0.3 * np.sin(0.3 * xx + 0.2 * yy) + 0.05 * rng.normal(size=(ny, nx)),
                        0.25 * np.cos(0.25 * xx - 0.4 * yy) + 0.05 * rng.normal(size=(ny, nx))), axis=-1)
        dt = 0.6 * min(dom.dx, dom.dy)
        data[f"adv_{tag}_in"] = vel
        data[f"adv_{tag}_sl"] = grid_mod.advect_velocity(vel, dt, dom, False)
        data[f"adv_{tag}_mc"] = grid_mod.advect_velocity(vel, dt, dom, True)
        data[f"adv_{tag}_in32"] = vel.astype(np.float32)
        data[f"adv_{tag}_mc32"] = grid_mod.advect_velocity(vel.astype(np.float32), dt, dom, True)
        meta[f"adv_{tag}"] = {"bounds": [list(b) for b in dom.bounds], "resolution": list(dom.resolution),
                              "periodic_axes": list(dom.periodic_axes), "dt": dt}
        # viscosity
        nu, ddt = 0.01, 0.02
        dvel, rep = grid_mod.implicit_diffuse(vel, nu, ddt, dom, 1.0e-9, 640)
        data[f"dif_{tag}_out"] = dvel
        meta[f"dif_{tag}"] = {"nu": nu, "dt": ddt, "tol": 1.0e-9, "iterations": rep.iterations,
                              "residual": rep.final_residual}
    # Poisson: DST preconditioned with a solid block, then periodic-x (Jacobi), then singular periodic
    for tag, shape, periodic, tol in (("dst", (32, 64), (), 1.0e-8), ("dst_odd", (27, 45), (), 1.0e-6),
                                      ("jac_x", (24, 40), ("x",), 1.0e-8), ("jac_xy", (16, 24), ("x", "y"), 1.0e-9)):
        ny, nx = shape
        rhs = rng.normal(size=shape)
        fluid = np.ones(shape, dtype=bool)
        fluid[ny // 3: ny // 2, nx // 3: nx // 2] = False
        dx, dy = 2.0 / nx, 1.2 / ny
        p, info, iters, rel = solve_masked_poisson(rhs.copy(), fluid, dx, dy, periodic, tol, 640)
        data[f"poi_{tag}_rhs"] = rhs
        data[f"poi_{tag}_fluid"] = fluid
        data[f"poi_{tag}_p"] = p
        meta[f"poi_{tag}"] = {"dx": dx, "dy": dy, "periodic_axes": list(periodic), "tol": tol, "info": info,
                              "iterations": iters, "relative_residual": rel}
    # DST-I at the call site's transform (scipy.fft.dstn type 1, ortho)
    from scipy.fft import dstn

    x = rng.normal(size=(9, 14))
    data["dst_in"] = x
    data["dst_out"] = dstn(x, type=1, norm="ortho")
    # face projection with a solid block (the reference unit test's set-up, seeded)
    dom = DomainSpec(2, ((-2.0, 2.0), (-1.0, 1.0)), (64, 32))
    vel = rng.normal(0.0, 0.1, (32, 64, 2))
    vel[:, :, 0] += 1.0
    solid = np.zeros((32, 64), dtype=bool)
    solid[12:20, 28:36] = True
    wall = np.zeros_like(vel)
    u, v = grid_mod.cell_to_faces(vel)
    data["prj_u_in"], data["prj_v_in"], data["prj_solid"] = u.copy(), v.copy(), solid
    pu, pv, rep = grid_mod.project_faces(u, v, dom, solid, wall, (1.0, 0.0), 0.01, False, 1.0e-9, 640)
    data["prj_u_out"], data["prj_v_out"] = pu, pv
    meta["prj"] = {"bounds": [list(b) for b in dom.bounds], "resolution": [64, 32], "dt": 0.01, "tol": 1.0e-9,
                   "iterations": rep.iterations, "relative_residual": rep.final_residual}
    data["meta"] = np.asarray(json.dumps(meta))
    np.savez_compressed(out / "operators.npz", **data)


def run_trajectory(M, grid_mod, sc, steps, out: Path, name: str, keep_every: bool = True,
                   dt_override=None, keep_steps=None) -> None:
    from foilbench_py.core.geometry import NacaFoil
    from foilbench_py.solvers.stable_fluids import StableFluidsSolver

    seen = {"pressure": None, "iters": []}
    original = grid_mod.solve_masked_poisson

    def recording(*args, **kwargs):
        p, info, iters, rel = original(*args, **kwargs)
        seen["pressure"] = p.copy()
        seen["iters"].append(int(iters))
        return p, info, iters, rel

    grid_mod.solve_masked_poisson = recording
    try:
        solver = StableFluidsSolver()
        solver.initialize(sc, NacaFoil(sc.foil), sc.seed)
        data = {"u0": solver._u.copy(), "v0": solver._v.copy(), "solid0": solver._solid.copy(),
                "p0": seen["pressure"].copy()}
        evid = [{"init_pressure_iterations": seen["iters"][-1]}]
        dt = dt_override if dt_override is not None else sc.output_dt
        for k in range(steps):
            seen["iters"] = []
            rep = solver.advance(sc.control_at((k + 1) * dt), dt)
            e = {key: (bool(val) if isinstance(val, (bool, np.bool_)) else float(val))
                 for key, val in rep.evidence.items()}
            e["substeps"] = rep.substeps
            e["max_speed"] = rep.max_speed
            e["projection_iterations"] = list(seen["iters"])
            e["angle_degrees"] = solver._control.angle_degrees
            e["angular_velocity_degrees"] = solver._control.angular_velocity_degrees
            evid.append(e)
            if keep_every or k == steps - 1 or (keep_steps is not None and k + 1 in keep_steps):
                data[f"u{k + 1}"] = solver._u.copy()
                data[f"v{k + 1}"] = solver._v.copy()
                data[f"p{k + 1}"] = seen["pressure"].copy()
        data["solid_final"] = solver._solid.copy()
        data["export"] = solver.export_state().velocity[0].copy()
        diag = solver.diagnostics().values
        data["diagnostics"] = np.asarray(json.dumps({k: float(v) for k, v in diag.items()}))
        data["scenario"] = np.asarray(json.dumps(scenario_dict(sc)))
        data["evidence"] = np.asarray(json.dumps(evid))
        data["meta"] = np.asarray(json.dumps({"steps": steps, "dt": dt, "keep_every": keep_every,
                                              "keep_steps": sorted(keep_steps) if keep_steps else None}))
        np.savez_compressed(out / f"traj_{name}.npz", **data)
    finally:
        grid_mod.solve_masked_poisson = original


def gen_trajectories(M, grid_mod, out: Path) -> None:
    c1_bounds = ((-1.0, 3.0), (-1.0, 1.0))
    sl = {"stable_advection": "semi-lagrangian", "stable_cfl": 0.5}
    # C1-shaped (NACA 0012 @ 8 deg, Re 1000, SL, CFL 0.5, FP64), reduced and full size
    run_trajectory(M, grid_mod, make_scenario(M, sid="c1-64x32", bounds=c1_bounds, resolution=(64, 32),
                                              naca="0012", angle=8.0, re=1000.0, precision="float64",
                                              options=sl, output_dt=0.5 * 4.0 / 64), 12, out, "c1_64x32")
    run_trajectory(M, grid_mod, make_scenario(M, sid="c1-64x32-tight", bounds=c1_bounds, resolution=(64, 32),
                                              naca="0012", angle=8.0, re=1000.0, precision="float64",
                                              options={**sl, "pressure_tolerance": 1.0e-10},
                                              output_dt=0.5 * 4.0 / 64), 8, out, "c1_64x32_tight")
    # C2-shaped (NACA 2412 @ 15 deg, Re 5000, tol 1e-6), reduced size, both precisions
    for prec in ("float64", "float32"):
        run_trajectory(M, grid_mod, make_scenario(M, sid=f"c2-128x64-{prec}", bounds=c1_bounds,
                                                  resolution=(128, 64), naca="2412", angle=15.0, re=5000.0,
                                                  precision=prec,
                                                  options={**sl, "pressure_tolerance": 1.0e-6},
                                                  output_dt=0.5 * 4.0 / 128), 6, out, f"c2_128x64_{prec}")
    # reference test helper: FP32 MacCormack NACA 2412 pitching 4 -> 20 deg (moving wall)
    helper_opts = {"initial_condition": "freestream", "pic_flip_blend": 0.95, "stable_advection": "maccormack"}
    run_trajectory(M, grid_mod, make_scenario(M, sid="helper", bounds=((-2.0, 6.0), (-2.0, 2.0)),
                                              resolution=(48, 24), naca="2412", angle=4.0, re=500.0,
                                              precision="float32", options=helper_opts,
                                              controls=[(0.0, 4.0), (1.0, 20.0)], output_dt=0.01), 6, out,
                   "helper_48x24")
    run_trajectory(M, grid_mod, make_scenario(M, sid="helper64", bounds=((-2.0, 6.0), (-2.0, 2.0)),
                                              resolution=(64, 32), naca="2412", angle=4.0, re=500.0,
                                              precision="float64", options=helper_opts,
                                              controls=[(0.0, 4.0), (0.2, 20.0)], output_dt=0.02), 6, out,
                   "pitch_64x32")
    # fixed stall (MacCormack, CFL 1.25, tol 1e-3), reduced
    stall = {"mac_maximum_divergence_linf": 2.25, "mac_maximum_solid_leakage": 0.0001,
             "pressure_tolerance": 0.001, "stable_advection": "maccormack", "stable_cfl": 1.25}
    run_trajectory(M, grid_mod, make_scenario(M, sid="stall", bounds=((-1.5, 3.5), (-1.5, 1.5)),
                                              resolution=(80, 48), naca="2412", angle=25.0, re=1000.0,
                                              precision="float32", options=stall,
                                              output_dt=0.016666666666666666), 5, out, "stall_80x48")
    # periodic validation flows
    run_trajectory(M, grid_mod, make_scenario(M, sid="taylor-green", bounds=((0.0, 6.283185307179586),
                                                                              (0.0, 6.283185307179586)),
                                              resolution=(32, 32), naca="0012", angle=0.0, re=100.0,
                                              precision="float64", options={"initial_condition": "taylor-green"},
                                              periodic=("x", "y"), pivot=(-10.0, -10.0), chord=0.2,
                                              freestream=(0.0, 0.0), output_dt=0.02), 5, out, "taylor_green_32")
    run_trajectory(M, grid_mod, make_scenario(M, sid="poiseuille", bounds=((0.0, 4.0), (-1.0, 1.0)),
                                              resolution=(48, 24), naca="0012", angle=0.0, re=100.0,
                                              precision="float64", options={"initial_condition": "poiseuille"},
                                              periodic=("x",), pivot=(-10.0, -10.0), chord=0.2,
                                              output_dt=0.02), 5, out, "poiseuille_48x24")


def gen_transport_trajectories(M, grid_mod, out: Path) -> None:
    """Opt-in transports: face-centred MacCormack / semi-Lagrangian (stable_face_advection) and
    skew-symmetric RK2 convection (stable_advection = skew-rk2)."""
    c1_bounds = ((-1.0, 3.0), (-1.0, 1.0))
    run_trajectory(M, grid_mod, make_scenario(M, sid="face-mc", bounds=c1_bounds, resolution=(64, 32), naca="2412",
                                              angle=10.0, re=500.0, precision="float64",
                                              options={"stable_face_advection": True, "stable_advection": "maccormack",
                                                       "stable_cfl": 0.5},
                                              output_dt=0.5 * 4.0 / 64), 5, out, "face_mc_64x32")
    run_trajectory(M, grid_mod, make_scenario(M, sid="face-sl", bounds=c1_bounds, resolution=(48, 24), naca="0012",
                                              angle=6.0, re=300.0, precision="float32",
                                              options={"stable_face_advection": True,
                                                       "stable_advection": "semi-lagrangian", "stable_cfl": 0.5},
                                              output_dt=0.5 * 4.0 / 48), 5, out, "face_sl_48x24")
    run_trajectory(M, grid_mod, make_scenario(M, sid="skew", bounds=c1_bounds, resolution=(64, 32), naca="2412",
                                              angle=12.0, re=800.0, precision="float64",
                                              options={"stable_advection": "skew-rk2", "stable_cfl": 0.5},
                                              output_dt=0.5 * 4.0 / 64), 5, out, "skew_64x32")
    run_trajectory(M, grid_mod, make_scenario(M, sid="skew-f32", bounds=c1_bounds, resolution=(48, 24), naca="0012",
                                              angle=5.0, re=400.0, precision="float32",
                                              options={"stable_advection": "skew-rk2", "stable_cfl": 0.5},
                                              output_dt=0.5 * 4.0 / 48), 5, out, "skew_48x24")


def gen_horizons(M, grid_mod, out: Path) -> None:
    """The configurations' own horizons: C1 (256x128 NACA 0012 at 8 deg, Re 1000) for its 200
    advances; C2 physics (NACA 2412 at 15 deg, Re 5000, tol 1e-6) in FP64 for 50 advances at
    256x128 with fields at steps 1, 10, 25 and 50, and one advance at the full 2048x1024 size
    summarised."""
    from foilbench_py.core.geometry import NacaFoil
    from foilbench_py.solvers.stable_fluids import StableFluidsSolver

    c1_bounds = ((-1.0, 3.0), (-1.0, 1.0))
    # the full C1 configuration: 200 advances from the freestream start, fields every 50
    run_trajectory(M, grid_mod, make_scenario(M, sid="c1-256x128", bounds=c1_bounds, resolution=(256, 128),
                                              naca="0012", angle=8.0, re=1000.0, precision="float64",
                                              options={"stable_advection": "semi-lagrangian", "stable_cfl": 0.5},
                                              output_dt=0.5 * 4.0 / 256), 200, out, "c1_256x128",
                   keep_every=False, keep_steps={1, 50, 100, 150, 200})
    sl = {"stable_advection": "semi-lagrangian", "stable_cfl": 0.5, "pressure_tolerance": 1.0e-6}
    run_trajectory(M, grid_mod, make_scenario(M, sid="c2-256x128-float64", bounds=c1_bounds, resolution=(256, 128),
                                              naca="2412", angle=15.0, re=5000.0, precision="float64", options=sl,
                                              output_dt=0.5 * 4.0 / 256), 50, out, "c2_256x128_float64",
                   keep_every=False, keep_steps={1, 10, 25, 50})
    sc = make_scenario(M, sid="c2-2048x1024-float64", bounds=c1_bounds, resolution=(2048, 1024), naca="2412",
                       angle=15.0, re=5000.0, precision="float64", options=sl, output_dt=0.5 * 4.0 / 2048)
    seen = {"pressure": None, "iters": []}
    original = grid_mod.solve_masked_poisson

    def recording(*args, **kwargs):
        p, info, iters, rel = original(*args, **kwargs)
        seen["pressure"] = p.copy()
        seen["iters"].append(int(iters))
        return p, info, iters, rel

    def summary(prefix, data, u, v, p):
        for key, a in (("u", u), ("v", v), ("p", p)):
            data[f"{prefix}_{key}_rows"] = a.sum(axis=1)
            data[f"{prefix}_{key}_cols"] = a.sum(axis=0)
            data[f"{prefix}_{key}_sub"] = a[::16, ::16].copy()
            data[f"{prefix}_{key}_norm"] = np.asarray(np.linalg.norm(a))

    grid_mod.solve_masked_poisson = recording
    try:
        solver = StableFluidsSolver()
        solver.initialize(sc, NacaFoil(sc.foil), sc.seed)
        data = {}
        summary("init", data, solver._u, solver._v, seen["pressure"])
        init_iters = seen["iters"][-1]
        seen["iters"] = []
        rep = solver.advance(sc.control_at(sc.output_dt), sc.output_dt)
        summary("step1", data, solver._u, solver._v, seen["pressure"])
        ev = {key: (bool(val) if isinstance(val, (bool, np.bool_)) else float(val)) for key, val in rep.evidence.items()}
        ev.update({"substeps": rep.substeps, "projection_iterations": list(seen["iters"]),
                   "init_pressure_iterations": init_iters})
        data["solid_count"] = np.asarray(int(solver._solid.sum()))
        data["scenario"] = np.asarray(json.dumps(scenario_dict(sc)))
        data["evidence"] = np.asarray(json.dumps(ev))
        np.savez_compressed(out / "c2full_2048x1024.npz", **data)
    finally:
        grid_mod.solve_masked_poisson = original


def gen_extras(M, grid_mod, out: Path) -> None:
    """sample_velocity (PY/solvers/stable_fluids.py:609-611) and restart (:218-236)."""
    from foilbench_py.core.geometry import NacaFoil
    from foilbench_py.core.models import RestartState
    from foilbench_py.solvers.stable_fluids import StableFluidsSolver

    c1_bounds = ((-1.0, 3.0), (-1.0, 1.0))
    sl = {"stable_advection": "semi-lagrangian", "stable_cfl": 0.5, "pressure_tolerance": 1.0e-10}
    data = {}
    meta = {}
    for prec in ("float64", "float32"):
        # float32 Jacobi viscosity (stopped by the pressure tolerance) cannot reach 1e-10
        opts = sl if prec == "float64" else {**sl, "pressure_tolerance": 1.0e-6}
        sc = make_scenario(M, sid=f"sample-{prec}", bounds=c1_bounds, resolution=(64, 32), naca="2412", angle=10.0,
                           re=800.0, precision=prec, options=opts, output_dt=0.5 * 4.0 / 64)
        solver = StableFluidsSolver()
        solver.initialize(sc, NacaFoil(sc.foil), 0)
        for k in range(3):
            solver.advance(sc.control_at((k + 1) * sc.output_dt), sc.output_dt)
        rng = np.random.default_rng(5)
        pts = np.concatenate([rng.uniform((-1.2, -1.2), (3.2, 1.2), (96, 2)),       # some outside the domain
                              rng.uniform((-0.1, -0.15), (1.0, 0.15), (32, 2)),     # near and inside the foil
                              np.asarray([[-1.0, -1.0], [3.0, 1.0], [1.0, 0.0]])])  # corners, a cell centre line
        data[f"sample_{prec}_points"] = pts
        data[f"sample_{prec}_values"] = np.asarray(solver.sample_velocity(pts))
        data[f"sample_{prec}_u"] = solver._u.copy()
        data[f"sample_{prec}_v"] = solver._v.copy()
        meta[f"sample_{prec}"] = scenario_dict(sc)
    # restart at a new pose and Reynolds number, then two advances toward a pitching control
    seen = {"pressure": None, "iters": []}
    original = grid_mod.solve_masked_poisson

    def recording(*args, **kwargs):
        p, info, iters, rel = original(*args, **kwargs)
        seen["pressure"] = p.copy()
        seen["iters"].append(int(iters))
        return p, info, iters, rel

    grid_mod.solve_masked_poisson = recording
    try:
        sc = make_scenario(M, sid="restart", bounds=c1_bounds, resolution=(64, 32), naca="4412", angle=4.0,
                           re=1000.0, precision="float64", options={**sl, "pressure_tolerance": 1.0e-9},
                           controls=[(0.0, 4.0), (2.0, 20.0)], output_dt=0.5 * 4.0 / 64)
        solver = StableFluidsSolver()
        start = RestartState(0.75, 12.0, 600.0)
        solver.restart(sc, NacaFoil(sc.foil), 0, start)
        data["restart_u0"], data["restart_v0"] = solver._u.copy(), solver._v.copy()
        data["restart_solid0"] = solver._solid.copy()
        data["restart_p0"] = seen["pressure"].copy()
        iters = [seen["iters"][-1]]
        for k in range(2):
            seen["iters"] = []
            t = start.time + (k + 1) * sc.output_dt
            c = sc.control_at(t)
            rep = solver.advance(c, sc.output_dt)
            data[f"restart_u{k + 1}"], data[f"restart_v{k + 1}"] = solver._u.copy(), solver._v.copy()
            iters.append({"substeps": rep.substeps, "pressure_iterations": list(seen["iters"])})
        meta["restart"] = {"scenario": scenario_dict(sc), "start": [start.time, start.angle_degrees, start.reynolds],
                           "evidence": iters}
    finally:
        grid_mod.solve_masked_poisson = original
    data["meta"] = np.asarray(json.dumps(meta))
    np.savez_compressed(out / "extras.npz", **data)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--only", default="")
    args = ap.parse_args()
    root = Path(args.reference)
    grid_mod = _import_reference(root)
    import foilbench_py.core.models as M

    out = HERE
    todo = args.only.split(",") if args.only else ["geometry", "masks", "operators", "trajectories"]
    if "geometry" in todo:
        gen_geometry(root, out)
    if "masks" in todo:
        gen_masks(out)
    if "operators" in todo:
        gen_operators(out, grid_mod)
    if "trajectories" in todo:
        gen_trajectories(M, grid_mod, out)
    if "trajectories" in todo or "transport" in todo:
        gen_transport_trajectories(M, grid_mod, out)
    if "trajectories" in todo or "horizons" in todo:
        gen_horizons(M, grid_mod, out)
    if "trajectories" in todo or "extras" in todo:
        gen_extras(M, grid_mod, out)
    print("golden fixtures written to", out)


if __name__ == "__main__":
    main()
