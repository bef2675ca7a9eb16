"""Where the FP32 error of the Stable Fluids step comes from: a CPU study on the oracle.

TEST INFRASTRUCTURE ONLY -- never imported by the product package.

Runs the oracle's FP64 restatement of the reference step (C2 physics: NACA 2412 at 15 deg,
Re 5000, semi-Lagrangian transport, CFL 0.5, pressure tolerance 1e-6) and variants that
round chosen stored arrays to float32 while keeping every operation in FP64, with the same
substep plan as the FP64 run, then prints the relative L2 errors of cell velocity and
pressure against the FP64 run at checkpoint steps:

  ref32  the reference's own float32 path (float32 arithmetic in every stencil)
  cells  cell planes rounded after faces->cells, advection and viscosity
  jcells cell planes rounded after faces->cells, advection and every Jacobi iteration
  faces  faces rounded after cells->faces and after the projection
  all    cells + faces (float32 storage of every velocity array, FP64 arithmetic)
  allJ   jcells + faces (what the mixed scheme's kernels do)

    python -m oracle.precision_study 256 100 ref32,all,allJ,faces

Pressure CG runs in FP64 throughout (as the reference runs it for float32 fields), so the
differences isolate the velocity storage and stencil arithmetic.
"""

from __future__ import annotations

import sys
import time

import numpy as np

from oracle import stable_fluids as O


def _scenario(nx: int, precision: str, tol: float):
    from foilbench_b200.workloads import single

    return single("precision-study", nx, nx // 2, "2412", 15.0, 5000.0, precision=precision, tolerance=tol)


def _r32(a):
    return a.astype(np.float32).astype(np.float64)


def _jacobi_rounded(vel, nu, dt, grid, tol, max_iter):
    """implicit_diffuse with every Jacobi iterate rounded to float32 (clamped edges)."""
    out, it, resid = [], 0, 0.0
    for c in range(vel.shape[2]):
        orig = vel[:, :, c].copy()
        cur = orig.copy()
        ax, ay = nu * dt / (grid.dx * grid.dx), nu * dt / (grid.dy * grid.dy)
        denom = 1.0 + 2.0 * ax + 2.0 * ay
        scale = max(float(np.max(np.abs(orig))), 1.0)
        for it in range(1, max_iter + 1):
            left = np.concatenate((cur[:, :1], cur[:, :-1]), axis=1)
            right = np.concatenate((cur[:, 1:], cur[:, -1:]), axis=1)
            down = np.concatenate((cur[:1, :], cur[:-1, :]), axis=0)
            up = np.concatenate((cur[1:, :], cur[-1:, :]), axis=0)
            nxt = _r32((orig + ax * (left + right) + ay * (down + up)) / denom)
            resid = float(np.max(np.abs(nxt - cur))) / scale
            cur = nxt
            if resid <= tol:
                break
        out.append(cur)
    return np.stack(out, axis=2), it, resid, True


def run(variant: str, nx: int, steps: int, tol: float, marks, plan=None):
    """One trajectory; returns ({step: (cell velocity, pressure)}, substep plan)."""
    sc = _scenario(nx, "float32" if variant == "ref32" else "float64", tol)
    s = O.OracleSolver(sc, keep_pressure=True)
    s.initialize()
    g = s.grid
    cells = variant in ("cells", "jcells", "all", "allJ")
    jac = variant in ("jcells", "allJ")
    faces = variant in ("faces", "all", "allJ")
    if faces:
        s.u, s.v = _r32(s.u), _r32(s.v)
    out, used = {}, []
    for k in range(steps):
        ctl = sc.control_at((k + 1) * sc.output_dt)
        if plan is None or variant == "ref32":
            rep = s.advance(ctl, sc.output_dt)
            used.append(rep.substeps)
        else:
            n = plan[k]
            dt = sc.output_dt / n
            nu = s.reference_speed * s.foil.chord / s.reynolds
            for _ in range(n):
                vel = O.faces_to_cell(s.u, s.v)
                vel = _r32(vel) if cells else vel
                vel = O.advect_velocity(vel, dt, g, False)
                vel = _r32(vel) if cells else vel
                if jac:
                    vel, _, _, _ = _jacobi_rounded(vel, nu, dt, g, tol, 640)
                else:
                    vel, _, _, _ = O.implicit_diffuse(vel, nu, dt, g, tol, 640)
                    vel = _r32(vel) if cells else vel
                s.u, s.v = O.cell_to_faces(vel)
                if faces:
                    s.u, s.v = _r32(s.u), _r32(s.v)
                keep = {}
                s.u, s.v, _ = O.project_faces(s.u, s.v, g, s.solid, s._wall(0.0), sc.freestream, dt, False, tol,
                                              640, keep)
                s.pressure = keep["pressure"]
                if faces:
                    s.u, s.v = _r32(s.u), _r32(s.v)
        if k + 1 in marks:
            out[k + 1] = (s.cell_velocity().astype(np.float64), np.asarray(s.pressure, dtype=np.float64))
    return out, used


def main(argv) -> None:
    nx, steps = int(argv[1]), int(argv[2])
    variants = argv[3].split(",")
    tol = float(argv[4]) if len(argv) > 4 else 1e-6
    marks = {k for k in (1, 10, 25, 50, 100, 150, 200, 300, 400) if k <= steps} | {steps}
    t0 = time.time()
    ref, plan = run("fp64", nx, steps, tol, marks)
    print(f"fp64 {nx}x{nx // 2}: {sum(plan)} substeps in {steps} steps ({time.time() - t0:.0f} s)", flush=True)
    for var in variants:
        got, _ = run(var, nx, steps, tol, marks, plan)
        for k in sorted(got):
            (vr, pr), (vg, pg) = ref[k], got[k]
            ev = np.linalg.norm(vg - vr) / np.linalg.norm(vr)
            ep = np.linalg.norm(pg - pr) / np.linalg.norm(pr)
            print(f"{var:7s} step {k:4d}  velocity {ev:.2e}  pressure {ep:.2e}", flush=True)


if __name__ == "__main__":
    main(sys.argv)
