#!/usr/bin/env python
"""Stable Fluids step benchmark on B200: MAC cell-steps/s (nx * ny * substeps / s).

Default workload (one GPU): 2048x1024 MAC grid on a 4x2-chord domain, NACA 2412 at 15 deg
(stall), Re 5000, float32 fields, semi-Lagrangian transport at CFL 0.5 (dt = 0.5 h), pressure
CG in FP32 inside an FP64 defect-correction loop to relative residual 1e-6. A "step" is one
``advance`` of one output interval (all its substeps); the state stays resident on the GPU.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c2|c2-fp64|c1|c5|c5-fp64]
    python bench.py --impl reference ...   # the reference algorithm on the host cores (CPU port)
    python bench.py --trace --workload c2 --steps 2   # per-phase device time of the step kernel

N > 1 (torchrun, one rank per GPU) runs independent replicas of the single-grid workload
(a single solve does not shard), so per-GPU work is fixed: "scaling": "weak".
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "MAC cell-steps/s"
FALLBACK_HBM_GBS = 6650.0

WORKLOADS = {
    "c2": dict(name="naca2412-15deg-Re5000-2048x1024-fp32-fp64dc", nx=2048, ny=1024, naca="2412", angle=15.0,
               re=5000.0, precision="float32", tol=1e-6, scheme="mixed", transport="semi-lagrangian"),
    "c2-fp64": dict(name="naca2412-15deg-Re5000-2048x1024-fp64-plain", nx=2048, ny=1024, naca="2412", angle=15.0,
                    re=5000.0, precision="float64", tol=1e-6, scheme="reference", transport="semi-lagrangian"),
    # C2's physics on a 4x larger grid, whose Krylov working set (235 MB) exceeds the 126 MB L2:
    # the case the step kernel's DRAM traffic is captured on
    "c2-4096": dict(name="naca2412-15deg-Re5000-4096x2048-fp32-fp64dc", nx=4096, ny=2048, naca="2412", angle=15.0,
                    re=5000.0, precision="float32", tol=1e-6, scheme="mixed", transport="semi-lagrangian"),
    "c1": dict(name="naca0012-8deg-Re1000-256x128-fp64-plain", nx=256, ny=128, naca="0012", angle=8.0, re=1000.0,
               precision="float64", tol=1e-5, scheme="reference", transport="semi-lagrangian"),
    "c5": dict(name="naca0012-10deg-Re1e4-8192x4096-fp32-200cg-scalar", nx=8192, ny=4096, naca="0012", angle=10.0,
               re=1.0e4, precision="float32", tol=1e-6, scheme="mixed", transport="semi-lagrangian", fixed=200,
               scalar=True),
    # C5 on the plain FP64 path (its comparator): rows of 8192 points as two half convolutions
    "c5-fp64": dict(name="naca0012-10deg-Re1e4-8192x4096-fp64-plain-200cg-scalar", nx=8192, ny=4096, naca="0012",
                    angle=10.0, re=1.0e4, precision="float64", tol=1e-6, scheme="reference",
                    transport="semi-lagrangian", fixed=200, scalar=True),
}


ROW_TRANSFORM = None  # --row-transform: the mixed scheme's preconditioner row DST (None: library default)


def make_scenario(w: dict):
    from foilbench_b200.models import ControlKeyframe, DomainSpec, FoilSpec, Scenario

    h = min(4.0 / w["nx"], 2.0 / w["ny"])
    opts = {"stable_advection": w["transport"], "stable_cfl": 0.5, "pressure_tolerance": w["tol"],
            "pressure_scheme": w["scheme"]}
    if w.get("fixed"):
        opts["pressure_fixed_iterations"] = int(w["fixed"])
        opts["pressure_max_iterations"] = max(640, 4 * int(w["fixed"]))
    if w.get("scalar"):
        opts["passive_scalar"] = True
    if ROW_TRANSFORM is not None and w["scheme"] == "mixed":
        opts["pressure_row_transform"] = ROW_TRANSFORM
    return Scenario(1, w["name"], DomainSpec(2, ((-1.0, 3.0), (-1.0, 1.0)), (w["nx"], w["ny"])), w["re"], (1.0, 0.0),
                    FoilSpec(w["naca"], 1.0, (0.0, 0.0)), (ControlKeyframe(0.0, w["angle"]),), 1.0e3, 0.5 * h,
                    w["precision"], 0, opts)


# ------------------------------------------------------------------------------- bytes model
def algorithmic_bytes_per_cell_substep(precision: str, scheme: str, n_visc: float, n_cg: float,
                                       scalar: bool = False) -> float:
    """The roofline's byte model: each stage separated by a global reduction or barrier reads
    and writes its live arrays once. In 4-byte words: advection 16 B, Jacobi 24 B per
    iteration, cells to faces / boundaries / right-hand side 20 B, per CG iteration 72 B
    (two row transforms 32 B, direction update with the operator and its dot 16 B, x/r update
    with the norm 24 B), true residual 8 B, gradient / boundaries / postconditions 20 B:
    B = 64 + 24 n_v + 72 n_cg (+ 8 for a passive scalar), velocity terms scaled by the field
    word and CG terms by the Krylov word (both 8 B in FP64: B_fp64 = 2 B_fp32)."""
    v = 8 if precision == "float64" else 4
    p = 4 if scheme == "mixed" else 8
    return (64 + 24 * n_visc) * v / 4 + 72 * n_cg * p / 4 + (8 if scalar else 0)


def bytes_per_cell_substep(precision: str, scheme: str, n_visc: float, n_cg: float, n_outer: float,
                           scalar: bool = False) -> float:
    """Bytes per cell and substep that the step as implemented moves when every stage reads
    and writes its live arrays once: beyond algorithmic_bytes_per_cell_substep it counts the
    solid mask (1 byte per read), the FP64 right-hand side, pressure and defect residual of the
    mixed scheme, the z and p reads of the CG direction update at their own stage, and the
    defect corrections. Reported beside the roofline, not used for its fraction.

    v = velocity word, p = Krylov word:
      faces->cells 4v | advection 4v + 1 | Jacobi 6v per iteration | cells->faces 4v
      | boundary copy 4v + 1 | divergence->RHS 2v + 1 + 16 | residual 17 | gradient 6v + 9
      | per CG iteration 16p + 3 (update+row DST) + 2p (column solve) + 3p + 1 (row DST)
        + 4p + 1 (p update, A p) = 25p + 5 | mixed: 16 for r64 = b, 8 + 4p + 25 per outer
        correction.
    """
    v = 8 if precision == "float64" else 4
    p = 4 if scheme == "mixed" else 8
    b = 4 * v + (4 * v + 1) + 6 * v * n_visc + 4 * v + (4 * v + 1) + (2 * v + 17) + 17 + (6 * v + 9)
    b += (25 * p + 5) * n_cg
    if scheme == "mixed":
        b += 16 + (33 + 4 * p) * n_outer
    if scalar:
        b += 3 * v
    return float(b)


# ------------------------------------------------------------------------------- clocks
class ClockSampler:
    """SM clocks and clock-event reasons of this process's GPU during the timed region: NVML
    read every 10 ms from a thread (the GPU matched by UUID, so a CUDA_VISIBLE_DEVICES mapping
    does not matter), else nvidia-smi every 200 ms. Reads only; no setting is changed."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.thread = None
        self.rows = []
        self.stop_flag = threading.Event()
        self.path = Path(tempfile.mkstemp(prefix="fb_clocks_", suffix=".csv")[1])

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        uuid = str(torch.cuda.get_device_properties(self.index).uuid)
        if not uuid.startswith("GPU-"):
            uuid = "GPU-" + uuid
        return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid)

    def _poll(self, nv, h):
        smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while not self.stop_flag.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((float(sm), float(smax), int(bits)))
            except Exception:
                pass
            self.stop_flag.wait(0.01)

    def start(self):
        try:
            nv, h = self._nvml_handle()
            self.thread = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None

    def stop(self) -> dict:
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join(timeout=5)
            if not self.rows:
                return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0, "source": "nvml"}
            reasons = sorted({name for _, _, bits in self.rows for name, bit in self.REASONS if bits & bit})
            return {"sm_mhz": statistics.median(r[0] for r in self.rows), "sm_max_mhz": max(r[1] for r in self.rows),
                    "reasons": reasons, "samples": len(self.rows), "source": "nvml, 10 ms"}
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        rows = []
        try:
            for line in self.path.read_text().splitlines():
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except OSError:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows), "source": "nvidia-smi, 200 ms"}


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
        except Exception:
            pass
    return {"hbm_gbs": FALLBACK_HBM_GBS, "source": "fallback"}


def _profile_value(name: str, key: str):
    p = ROOT / "profiles" / f"step_kernel_{name}.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith(key + ":"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


# workloads too large for a capture under the profiling size rule take the DRAM-to-algorithmic
# byte ratio of the same step kernel on a grid whose working set also exceeds L2
TRAFFIC_SCALED_FROM = {"c5": "c2-4096"}


def profiled_traffic(workload: str, algo_bytes: float):
    """DRAM bytes per step-kernel launch from the committed ncu summary of this workload, or
    scaled from another workload's capture by algorithmic bytes; (bytes, how) or (None, why)."""
    own = _profile_value(workload, "dram_bytes_per_launch")
    if own is not None:
        return own, f"ncu capture of this workload (profiles/step_kernel_{workload}.txt)"
    src = TRAFFIC_SCALED_FROM.get(workload)
    if src:
        t, a = _profile_value(src, "dram_bytes_per_launch"), _profile_value(src, "algorithmic_bytes_per_launch")
        if t and a:
            return t / a * algo_bytes, (f"scaled: DRAM/algorithmic ratio {t / a:.3f} of the {src} capture "
                                        f"(profiles/step_kernel_{src}.txt) times this launch's algorithmic bytes")
    return None, "no DRAM capture for this workload"


def limiter_note(traffic, algo_bytes, per_launch_s: float, peak_gbs: float) -> str:
    """What bounds the step kernel, from the profiled DRAM traffic per launch against the
    algorithmic bytes and against the HBM peak (the roofline's denominator either way)."""
    if not traffic:
        return "no DRAM capture for this workload"
    r = traffic / algo_bytes
    bw = traffic / per_launch_s / 1e9
    if r < 0.5:
        return (f"DRAM moves {r:.2f} of the algorithmic bytes: the Krylov working set is L2-resident, so HBM does "
                "not bind; the step is bound by latency and instruction issue")
    if bw < 0.5 * peak_gbs:
        return (f"DRAM moves {r:.2f} of the algorithmic bytes (operands stream about once) at {bw:.0f} GB/s, "
                f"{bw / peak_gbs:.2f} of peak: bound by latency and instruction issue, not by HBM bandwidth")
    return f"DRAM moves {r:.2f} of the algorithmic bytes at {bw:.0f} GB/s: HBM bandwidth binds"


# ------------------------------------------------------------------------------- CPU legs
# Above this many cells one advance of the CPU port runs for over an hour (C5: 8192x4096 with
# 200 CG sweeps per substep), so its sample is formed from timed parts of one substep.
PARTS_LIMIT_CELLS = 8_000_000


def cpu_sample_parts(workload: str) -> dict:
    """Bounded CPU sample of one substep of a very large workload: the port's own functions run
    once each on the workload's start state (transport, viscosity, mask), the projection once
    with 1 and once with 2 CG sweeps; one substep = transport + viscosity + mask + projection
    set-up + sweeps x (time per sweep), with the workload's sweep count."""
    import numpy as np

    from oracle.stable_fluids import (OracleSolver, advect_scalar, advect_velocity, cell_to_faces, faces_to_cell,
                                      implicit_diffuse, project_faces)

    w = WORKLOADS[workload]
    sc = make_scenario(w)
    o = OracleSolver(sc)
    g = o.grid
    c0 = sc.control_at(0.0)
    u, v = cell_to_faces(o._initial_velocity())
    dt = sc.output_dt
    nu = o.reference_speed * o.foil.chord / float(sc.reynolds)
    tol = float(w["tol"])
    clock = time.perf_counter
    t0 = clock()
    vel = faces_to_cell(u, v)
    if w.get("scalar"):
        advect_scalar(np.zeros(vel.shape[:2], dtype=vel.dtype), vel, dt, g)
    vel = advect_velocity(vel, dt, g, w["transport"] == "maccormack")
    t_adv = clock() - t0
    t0 = clock()
    vel, _, _, _ = implicit_diffuse(vel, nu, dt, g, tol, 640)
    uu, vv = cell_to_faces(vel)
    t_visc = clock() - t0
    t0 = clock()
    solid = o._mask(c0.angle_degrees)
    t_mask = clock() - t0
    wall = o._wall(0.0)
    proj = {}
    for k in (1, 2):
        t0 = clock()
        project_faces(uu.copy(), vv.copy(), g, solid, wall, sc.freestream, dt, False, tol, k, None)
        proj[k] = clock() - t0
    per_sweep = proj[2] - proj[1]
    setup = max(proj[1] - per_sweep, 0.0)
    sweeps = int(w.get("fixed") or 0)
    if sweeps <= 0:
        raise RuntimeError("the parts sample needs a fixed CG sweep count")
    substep = t_adv + t_visc + t_mask + setup + sweeps * per_sweep
    sampled = t_adv + t_visc + t_mask + proj[1] + proj[2]
    return {"cell_substeps": w["nx"] * w["ny"], "seconds": substep, "advances": 0,
            "sample": (f"one substep formed from timed parts ({sampled:.0f} s of CPU time): transport "
                       f"{t_adv:.1f} s, viscosity {t_visc:.1f} s, mask {t_mask:.1f} s, projection set-up "
                       f"{setup:.1f} s, {sweeps} CG sweeps x {per_sweep:.2f} s (timed over 1 and 2 sweeps); "
                       "numpy restatement of the reference path, one core")}


def cpu_sample(workload: str, advances: int) -> dict:
    """Run the CPU oracle (numpy restatement of the reference path) for a bounded sample."""
    from oracle.stable_fluids import OracleSolver

    w = WORKLOADS[workload]
    if w["nx"] * w["ny"] > PARTS_LIMIT_CELLS:
        return cpu_sample_parts(workload)
    sc = make_scenario(w)
    o = OracleSolver(sc)
    o.initialize()
    cells = w["nx"] * w["ny"]
    tot, subs = 0.0, 0
    for k in range(advances):
        c = sc.control_at((k + 1) * sc.output_dt)
        t0 = time.perf_counter()
        st = o.advance(c, sc.output_dt)
        tot += time.perf_counter() - t0
        subs += st.substeps
    return {"cell_substeps": cells * subs, "seconds": tot, "advances": advances}


def cpu_sample_subprocess(workload: str, advances: int, procs: int) -> dict:
    cmds = [[sys.executable, str(Path(__file__).resolve()), "--cpu-sample", workload, "--cpu-advances", str(advances)]
            for _ in range(procs)]
    env = dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1", MKL_NUM_THREADS="1",
               CUDA_VISIBLE_DEVICES="")
    t0 = time.perf_counter()
    ps = [subprocess.Popen(c, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, env=env) for c in cmds]
    outs = []
    for p in ps:
        out, err = p.communicate(timeout=3600)
        if p.returncode != 0:
            raise RuntimeError(f"CPU sample failed: {err[-2000:]}")
        outs.append(json.loads(out.strip().splitlines()[-1]))
    wall = time.perf_counter() - t0
    cs = sum(o["cell_substeps"] for o in outs)
    busy = max(o["seconds"] for o in outs)
    return {"value": cs / busy, "cores": procs, "cell_substeps": cs, "advance_seconds": busy, "wall_s": wall,
            "sample": outs[0].get("sample")}


# ------------------------------------------------------------------------------- GPU arm
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    return world, rank, local


def reduce_max(value: float, world: int) -> float:
    from foilbench_b200.replicas import max_over_ranks

    return float(value) if world == 1 else max_over_ranks(value, device="cuda")


def barrier(world: int):
    import torch

    if world > 1:
        import torch.distributed as dist

        dist.barrier()
    torch.cuda.synchronize()


def run_gpu(args) -> dict | None:
    import numpy as np
    import torch

    world, rank, local = dist_setup(args)
    from foilbench_b200.geometry import NacaFoil
    from foilbench_b200.solver import StableFluidsSolver

    w = WORKLOADS[args.workload]
    sc = make_scenario(w)
    solver = StableFluidsSolver(device=local)
    solver.initialize(sc, NacaFoil(sc.foil), 0)
    dt = sc.output_dt
    step = [0]
    # launch shapes and sweep schedule by measurement on this grid (state unchanged; cached for
    # the later solvers of the same grid, the error-window runs included)
    tune = None if args.no_tune else solver.autotune(dt)

    def advance():
        step[0] += 1
        return solver.advance(sc.control_at(step[0] * dt), dt)

    for _ in range(args.warmup):
        advance()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    clocks = ClockSampler(local)
    barrier(world)
    clocks.start()
    t_wall0 = time.perf_counter()
    dev_ms, subs, launches, cg_total, reports = 0.0, 0, 0, 0, []
    for _ in range(args.steps):
        flush.zero_()  # evict L2 (256 MiB write) between timed steps; not inside any step's events
        torch.cuda.synchronize()
        rep = advance()
        ev = rep.evidence
        dev_ms += ev["device_ms"]
        subs += rep.substeps
        launches += ev["kernel_launches"]
        cg_total += ev["pressure_total_iterations"]
        reports.append(rep)
    barrier(world)
    wall = time.perf_counter() - t_wall0
    clk = clocks.stop()
    dev_ms_max = reduce_max(dev_ms, world)
    cells = w["nx"] * w["ny"]
    value = world * cells * subs / (dev_ms_max / 1e3)

    # roofline of the persistent step kernel (one launch per substep)
    last = reports[-1].evidence
    n_v = float(np.mean([r.evidence["viscosity_iterations"] for r in reports]))
    n_cg = cg_total / max(subs, 1)
    n_out = float(np.mean([r.evidence["pressure_outer_iterations"] for r in reports]))
    bpc = algorithmic_bytes_per_cell_substep(w["precision"], w["scheme"], n_v, n_cg, bool(w.get("scalar")))
    impl_bpc = bytes_per_cell_substep(w["precision"], w["scheme"], n_v, n_cg, n_out, bool(w.get("scalar")))
    per_launch_s = dev_ms / 1e3 / max(launches, 1)
    algo_bytes = bpc * cells
    achieved = algo_bytes / per_launch_s / 1e9
    peaks = measured_peaks()
    traffic, traffic_how = profiled_traffic(args.workload, algo_bytes)

    # end-to-end through the public API: control in, StepReport + canonical velocity out
    state_bytes = cells * 2 * (4 if w["precision"] == "float32" else 8)
    # warm-up of the end-to-end path: the exports' page-locked host blocks come from the
    # library's pool, which is filled here (two blocks are live at once in the loop below)
    warm = [solver.export_state(), solver.export_state()]
    del warm
    barrier(world)
    t0 = time.perf_counter()
    e2e_subs = 0
    for _ in range(args.steps):
        rep = advance()
        e2e_subs += rep.substeps
        _ = solver.export_state()
    barrier(world)
    e2e_wall = reduce_max(time.perf_counter() - t0, world)
    e2e_value = world * cells * e2e_subs / e2e_wall

    # the metric's comparator and this scheme's error against it over the error window (three
    # solves in lockstep over up to 200 steps: grids over 4096 columns, where one FP64 step
    # takes seconds, get the comparator only)
    fp64 = err = None
    if w["precision"] == "float32" and not args.no_fp64:
        fp64 = plain_fp64_comparator(args, local, flush)
        if w["nx"] <= 4096:
            err = error_vs_fp64(args.workload, local, args.error_steps)

    if rank != 0:
        return None
    out = {
        "metric": METRIC,
        "value": value,
        "unit": "cell-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": dev_ms_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32+f64" if w["scheme"] == "mixed" else ("f64" if w["precision"] == "float64" else "f32"),
        "data": "synthetic scenario (seeded, no dataset): freestream start, fixed foil pose",
        "config": {"workload": w["name"], "grid": f"{w['nx']}x{w['ny']}", "domain": "[-1,3]x[-1,1]",
                   "naca": w["naca"], "angle_deg": w["angle"], "reynolds": w["re"], "precision": w["precision"],
                   "pressure_scheme": w["scheme"], "pressure_tolerance": w["tol"], "transport": w["transport"],
                   "cfl": 0.5, "dt": dt, "substeps_per_step": subs / args.steps,
                   "cg_iterations_per_substep": n_cg, "jacobi_iterations": n_v, "defect_corrections": n_out,
                   "l2": "flushed between timed steps (256 MiB device write outside the step timing)",
                   "parallelism": f"replicas x{world}", "wall_ms_per_step": wall * 1e3 / args.steps,
                   "pressure_relative_residual": last["pressure_relative_residual"]},
        "roofline": {"bound": "hbm", "kernel": "fb::step_kernel", "achieved": achieved, "peak": peaks["hbm_gbs"],
                     "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
                     "algorithmic_bytes_per_launch": algo_bytes, "bytes_per_cell_substep": bpc,
                     "bytes_model": "64 + 24 n_v + 72 n_cg per cell-substep in 4-byte words (x2 for 8-byte words)",
                     "implementation_bytes_per_cell_substep": impl_bpc,
                     "traffic": traffic, "traffic_source": traffic_how,
                     "traffic_over_algorithmic": (traffic / algo_bytes) if traffic else None,
                     "limiter": limiter_note(traffic, algo_bytes, per_launch_s, peaks["hbm_gbs"])},
        "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": 32,
                "d2h_bytes_per_step": state_bytes + 256,
                "note": "StableFluidsSolver.advance(control) + export_state() per step through libfoilb200"},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if tune is not None:
        out["autotune"] = tune
    if fp64 is not None:
        out["plain_fp64_gpu"] = dict(fp64, ratio=value / fp64["value"])
    if err is not None:
        out["error_vs_fp64"] = err
    if world == 1 and not args.no_cpu:
        try:
            cb = cpu_sample_subprocess(args.workload, 1, 1)
            out["cpu_baseline"] = {"value": cb["value"], "unit": "cell-steps/s", "cores": 1, "kind": "port",
                                   "sample": cb.get("sample") or (
                                       f"1 advance of the same workload after initialisation "
                                       f"({cb['advance_seconds']:.1f} s of CPU time), numpy restatement of the "
                                       "reference path, float32 fields with FP64 CG as the reference runs them")}
        except Exception as err:  # pragma: no cover - reported, not fatal
            out["cpu_baseline"] = {"value": None, "unit": "cell-steps/s", "cores": 0, "kind": "port",
                                   "sample": f"failed: {err}"}
    return out


def _compare(a, b) -> dict:
    """Relative L2 / L-inf errors of solver a's fields against solver b's (the FP64 path)."""
    import numpy as np

    def div(sv):
        u, v = sv.face_velocities()
        sc = sv._scenario
        dx = (sc.domain.bounds[0][1] - sc.domain.bounds[0][0]) / sc.domain.nx
        dy = (sc.domain.bounds[1][1] - sc.domain.bounds[1][0]) / sc.domain.ny
        d = (np.diff(np.asarray(u, np.float64), axis=1) / dx + np.diff(np.asarray(v, np.float64), axis=0) / dy)
        d[sv.solid_mask()] = 0.0
        return d

    out = {}
    for name, x, y in (("velocity", a.cell_velocity(), b.cell_velocity()), ("pressure", a.pressure(), b.pressure()),
                       ("divergence", div(a), div(b))):
        d = np.asarray(x, dtype=np.float64) - y
        out[f"{name}_rel_l2"] = float(np.linalg.norm(d) / max(np.linalg.norm(y), 1e-300))
        out[f"{name}_rel_linf"] = float(np.abs(d).max() / max(np.abs(y).max(), 1e-300))
    fa, fb = a.forces(), b.forces()
    for k in ("lift_coefficient", "drag_coefficient"):
        out[k.split("_")[0] + "_coefficient_rel"] = abs(fa[k] - fb[k]) / max(abs(fb[k]), 1e-300)
    out["lift_coefficient"] = fa["lift_coefficient"]
    out["drag_coefficient"] = fa["drag_coefficient"]
    return out


ERROR_CHECKPOINTS = (1, 10, 25, 50, 100, 150, 200)


def error_vs_fp64(workload: str, device: int, horizon: int) -> dict:
    """Accuracy of the FP32 + FP64-refined fields against the plain FP64 GPU path (the
    reference's scheme in FP64, parity-tested against the reference) over the workload's error
    window: three solves of the same scenario advance in lockstep from initialisation (this
    workload's scheme, the FP64 path at this tolerance, and the FP64 path at 1e-10), and the
    fields are compared at each checkpoint step up to `horizon`. Reports the errors at the last
    checkpoint, their maximum over the window, and the FP64 path's own spread between this
    tolerance and 1e-10 (differences of that size come from where the pressure iteration stops,
    not from the arithmetic)."""
    from foilbench_b200.geometry import NacaFoil
    from foilbench_b200.solver import StableFluidsSolver

    def make(w):
        sc = make_scenario(w)
        sv = StableFluidsSolver(device=device)
        sv.initialize(sc, NacaFoil(sc.foil), 0)
        return sc, sv

    w = WORKLOADS[workload]
    w64 = dict(w, precision="float64", scheme="reference")
    sc, mixed = make(w)
    _, ref = make(w64)
    _, tight = make(dict(w64, tol=1e-10))
    marks = [k for k in ERROR_CHECKPOINTS if k <= horizon] or [horizon]
    window, spread_window, last, spread = {}, {}, None, None
    for k in range(1, max(marks) + 1):
        c = sc.control_at(k * sc.output_dt)
        for sv in (mixed, ref, tight):
            sv.advance(c, sc.output_dt)
        if k in marks:
            last = _compare(mixed, ref)
            spread = _compare(ref, tight)
            window[k] = last
            spread_window[k] = spread
    keys = ("velocity_rel_l2", "velocity_rel_linf", "pressure_rel_l2", "pressure_rel_linf", "divergence_rel_l2",
            "lift_coefficient_rel", "drag_coefficient_rel")
    out = {"after_steps": max(marks), "tolerance": w["tol"], **last,
           "max_over_window": {k: max(window[m][k] for m in marks) for k in keys},
           "checkpoints": {str(m): {k: window[m][k] for k in ("velocity_rel_l2", "pressure_rel_l2")} for m in marks},
           "fp64_tolerance_spread": {k: spread[k] for k in ("velocity_rel_l2", "pressure_rel_l2", "pressure_rel_linf",
                                                             "lift_coefficient_rel", "drag_coefficient_rel")},
           "fp64_tolerance_spread_max": {k: max(spread_window[m][k] for m in marks)
                                         for k in ("velocity_rel_l2", "pressure_rel_l2")},
           "comparator": "plain FP64 GPU path (float64 fields, the reference's FP64 CG) at the same tolerance"}
    for sv in (mixed, ref, tight):
        sv.close()
    return out


def plain_fp64_comparator(args, local: int, flush) -> dict:
    """The metric's comparator: the plain FP64 GPU drop-in (float64 fields, the reference's
    FP64 pressure CG) on the same scenario, timed like the headline over the same step indices
    (the same warm-up, then the same number of timed steps with L2 flushed in between)."""
    import torch

    from foilbench_b200.geometry import NacaFoil
    from foilbench_b200.solver import StableFluidsSolver

    w = dict(WORKLOADS[args.workload], precision="float64", scheme="reference")
    sc = make_scenario(w)
    sv = StableFluidsSolver(device=local)
    sv.initialize(sc, NacaFoil(sc.foil), 0)
    tune = None if args.no_tune else sv.autotune(sc.output_dt)
    k = 0
    for _ in range(args.warmup):
        k += 1
        sv.advance(sc.control_at(k * sc.output_dt), sc.output_dt)
    dev_ms, subs, cg = 0.0, 0, 0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        k += 1
        rep = sv.advance(sc.control_at(k * sc.output_dt), sc.output_dt)
        dev_ms += rep.evidence["device_ms"]
        subs += rep.substeps
        cg += rep.evidence["pressure_total_iterations"]
    sv.close()
    cells = w["nx"] * w["ny"]
    return {"value": cells * subs / (dev_ms / 1e3), "unit": "cell-steps/s", "ms_per_step": dev_ms / args.steps,
            "substeps_per_step": subs / args.steps, "cg_iterations_per_substep": cg / max(subs, 1),
            "autotune": tune,
            "how": "same scenario and step indices, float64 fields and the reference's FP64 CG (one solve), "
                   "launch shapes tuned the same way"}


def run_trace(args) -> None:
    """Per-phase device time of the step kernel (CTA 0 stamps %globaltimer after every grid
    barrier) over `--steps` advances after the warm-up; printed as a table, not a bench line."""
    from foilbench_b200.geometry import NacaFoil
    from foilbench_b200.solver import StableFluidsSolver

    w = WORKLOADS[args.workload]
    sc = make_scenario(w)
    solver = StableFluidsSolver()
    solver.initialize(sc, NacaFoil(sc.foil), 0)
    dt = sc.output_dt
    k = 0
    for _ in range(args.warmup):
        k += 1
        solver.advance(sc.control_at(k * dt), dt)
    solver.enable_trace(1 << 18)
    dev, subs, cg = [], [], []
    for _ in range(args.steps):
        k += 1
        rep = solver.advance(sc.control_at(k * dt), dt)
        dev.append(round(rep.evidence["device_ms"], 3))
        subs.append(rep.substeps)
        cg.append(rep.evidence["pressure_total_iterations"])
    summary = solver.trace_summary(solver.read_trace())
    total = sum(d["us"] for d in summary.values())
    print(f"== {args.workload}: device_ms {dev} substeps {subs} cg {cg} traced_us {total:.0f}")
    for name, d in sorted(summary.items(), key=lambda kv: -kv[1]["us"]):
        print(f"   {name:28s} {d['us']:11.1f} us  n={d['count']:5d}  per={d['us'] / max(d['count'], 1):9.2f} us")


def run_batched(args) -> dict:
    """C3: 64 seeded uneven scenarios advanced together, one batched launch per substep round.

    Also times the same scenarios as plain FP64 single solves (the reference's scheme in FP64,
    one solve at a time) and reports the velocity error of the batched FP32+FP64-refined
    fields against them after the same steps."""
    import numpy as np
    import torch

    from foilbench_b200 import workloads
    from foilbench_b200.batch import StableFluidsBatch
    from foilbench_b200.geometry import NacaFoil
    from foilbench_b200.models import NumericalFailure
    from foilbench_b200.solver import StableFluidsSolver

    from foilbench_b200.replicas import job_throughput, partition

    world, rank, local = dist_setup(args)
    everything = workloads.batched_mix(args.seed, args.batch_count)
    mine = partition([sc.domain.nx * sc.domain.ny for sc in everything], world)[rank]
    scs = [everything[i] for i in mine]
    solvers = []
    for sc in scs:
        s = StableFluidsSolver(device=local)
        s.initialize(sc, NacaFoil(sc.foil), 0)
        solvers.append(s)
    batch = StableFluidsBatch(solvers)
    step = [0]

    def batch_step():
        step[0] += 1
        reps = batch.advance([sc.control_at(step[0] * sc.output_dt) for sc in scs], [sc.output_dt for sc in scs])
        bad = [r for r in reps if isinstance(r, NumericalFailure)]
        if bad:
            raise RuntimeError(f"{len(bad)} batch members failed: {bad[0]}")
        return reps

    for _ in range(args.warmup):
        batch_step()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    clocks = ClockSampler(local)
    clocks.start()
    dev_ms, cs, launches, algo = 0.0, 0, 0, 0.0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        reps = batch_step()
        dev_ms += reps[0].evidence["device_ms"]
        launches += reps[0].evidence["kernel_launches"]
        cs += sum(sc.domain.nx * sc.domain.ny * r.substeps for sc, r in zip(scs, reps))
        # the roofline's byte model per member (its own Jacobi and CG counts)
        for sc, r in zip(scs, reps):
            ev = r.evidence
            n_cg = ev["pressure_total_iterations"] / max(r.substeps, 1)
            algo += sc.domain.nx * sc.domain.ny * r.substeps * algorithmic_bytes_per_cell_substep(
                "float32", "mixed", float(ev["viscosity_iterations"]), n_cg)
    clk = clocks.stop()
    value = job_throughput(cs, dev_ms / 1e3, device="cuda")
    # end to end: batched advance + every member's canonical velocity to the host
    t0 = time.perf_counter()
    e2e_cs, d2h = 0, 0
    for _ in range(args.steps):
        reps = batch_step()
        e2e_cs += sum(sc.domain.nx * sc.domain.ny * r.substeps for sc, r in zip(scs, reps))
        for s in solvers:
            d2h += s.export_state().velocity.nbytes
    e2e = job_throughput(e2e_cs, time.perf_counter() - t0, device="cuda")
    steps_done = step[0]
    # plain FP64 GPU path: the same scenarios, FP64 fields and the reference's FP64 CG, advanced
    # the same number of steps (also for the error comparison). Timed two ways: each solve alone
    # on the whole GPU, one after another; and each solve alone on the CTAs it has in the batched
    # launch, where the members of a batch run side by side, so the job time is the slowest one's.
    shares = batch.ctas() if batch._handle else [0] * len(scs)
    err_v, fp64_ms, fp64_cs, share_ms, share_cs = [], 0.0, 0, [], 0
    for sc, s, share in zip(scs, solvers, shares):
        sc64 = workloads.single(sc.id + "-fp64", sc.domain.nx, sc.domain.ny, sc.foil.naca,
                                sc.control_at(0.0).angle_degrees, sc.reynolds, precision="float64")
        r64 = StableFluidsSolver(device=local)
        r64.initialize(sc64, NacaFoil(sc64.foil), 0)
        q64 = StableFluidsSolver(device=local)
        q64.initialize(sc64, NacaFoil(sc64.foil), 0)
        if share > 0:
            q64.set_launch_shape(ctas=share)
        ms_here = 0.0
        for k in range(steps_done):
            c = sc64.control_at((k + 1) * sc64.output_dt)
            rep = r64.advance(c, sc64.output_dt)
            rq = q64.advance(c, sc64.output_dt)
            if k >= args.warmup:
                fp64_ms += rep.evidence["device_ms"]
                fp64_cs += sc.domain.nx * sc.domain.ny * rep.substeps
                ms_here += rq.evidence["device_ms"]
                share_cs += sc.domain.nx * sc.domain.ny * rq.substeps
        share_ms.append(ms_here)
        a = s.cell_velocity().astype(np.float64)
        b = r64.cell_velocity()
        err_v.append(float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)))
        r64.close()
        q64.close()
    share_value = job_throughput(share_cs, max(share_ms) / 1e3, device="cuda")
    fp64_value = job_throughput(fp64_cs, fp64_ms / 1e3, device="cuda")
    cells = [sc.domain.nx * sc.domain.ny for sc in scs]
    peaks = measured_peaks()
    ctas = batch_ctas_summary(batch)
    batch.close()
    if rank != 0:
        return None
    return {
        "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
        "scaling": "strong" if world > 1 else "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic scenarios (seeded, no dataset)",
        "config": {"workload": f"batched-{len(everything)}-uneven-seed{args.seed}",
                   "grids": "uniform over 256x128, 512x256, 768x384, 1024x512",
                   "cells_total": int(sum(sc.domain.nx * sc.domain.ny for sc in everything)),
                   "scenarios_on_rank0": len(scs),
                   "naca": "camber 0-4 %, thickness 9-18 %", "angle_deg": "U[-5, 20]", "reynolds": "10^U[2, 4]",
                   "precision": "float32", "pressure_scheme": "mixed", "pressure_tolerance": 1e-6,
                   "transport": "semi-lagrangian", "cfl": 0.5, "ctas_per_member": ctas,
                   "l2": "flushed between timed steps (256 MiB device write outside the step timing)",
                   "parallelism": "one batched cooperative launch per substep round"},
        "plain_fp64_gpu": {"value": share_value, "unit": "cell-steps/s", "ratio": value / share_value,
                           "how": "same scenarios, float64 fields and FP64 CG, each solve alone on the CTAs it has "
                                  "in the batched launch; job time = the slowest member's (members run side by side)",
                           "one_at_a_time": {"value": fp64_value, "ratio": value / fp64_value,
                                             "how": "each solve alone on the whole GPU, one after another"}},
        "error_vs_fp64": {"velocity_rel_l2_max": max(err_v), "velocity_rel_l2_median": float(np.median(err_v)),
                          "after_steps": steps_done},
        "roofline": {"bound": "hbm", "kernel": "fb::step_kernel_batch", "achieved": algo / (dev_ms / 1e3) / 1e9,
                     "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": algo / (dev_ms / 1e3) / 1e9 / peaks["hbm_gbs"], "traffic": None,
                     "algorithmic_bytes_per_launch": algo / max(launches, 1),
                     "bytes_model": "64 + 24 n_v + 72 n_cg per cell-substep in 4-byte words, each member with its "
                                    "own Jacobi and CG counts",
                     "traffic_source": "no DRAM capture of the batched launch"},
        "e2e": {"value": e2e, "unit": "cell-steps/s", "h2d_bytes_per_step": 32 * len(scs),
                "d2h_bytes_per_step": d2h // max(args.steps, 1)},
        "gpu_launches": launches, "clocks": clk,
    }


def batch_ctas_summary(batch) -> str:
    c = batch.ctas() if batch._handle else []
    return f"min {min(c)}, max {max(c)}, total {sum(c)}" if c else ""


def run_served(args) -> dict:
    """C4: Poisson arrivals (200/s over 60 s, steps U[100, 2000], scenarios as in C3) served by
    the continuous-batching loop under a 150 GB HBM budget, for a bounded wall-clock window."""
    from foilbench_b200 import workloads
    from foilbench_b200.serving import ServedSolves

    reqs = workloads.request_stream(args.seed, args.rate, args.duration)
    served = ServedSolves(hbm_budget=int(args.budget_gb * 1e9), max_members=args.batch_count, keep_fields=True)
    clocks = ClockSampler(0)
    clocks.start()
    t0 = time.perf_counter()
    stats = served.run(reqs, until_s=args.serve_seconds)
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    p = stats.latency_percentiles()
    done = [c for c in stats.completed if not c.failed]
    # offered work: every request's steps at its grid, at the substeps its solve plans (about
    # 2.5 per step at CFL 0.5; counted here as executed substeps per step of the served ones)
    by_id = {r.rid: r for r in reqs}
    grid_steps = sum(c.steps * by_id[c.rid].scenario.domain.nx * by_id[c.rid].scenario.domain.ny for c in done)
    sub_per_step = sum(c.cell_steps for c in done) / grid_steps if grid_steps else 2.5
    offered = sum(r.steps * r.scenario.domain.nx * r.scenario.domain.ny for r in reqs) * sub_per_step
    audit = audit_served(reqs, done)
    return {
        "metric": METRIC, "value": stats.executed_cell_steps / max(stats.device_s, 1e-9), "unit": "cell-steps/s",
        "n_gpus": 1, "steps": stats.ticks, "warmup": 0, "ms_per_step": 1e3 * stats.device_s / max(stats.ticks, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic request stream (seeded Poisson arrivals, no dataset)",
        "config": {"workload": f"served-poisson{args.rate:g}-per-s-{args.duration:g}s-seed{args.seed}",
                   "offered_requests": len(reqs), "window_s": args.serve_seconds, "hbm_budget_gb": args.budget_gb,
                   "max_members": args.batch_count,
                   "offered_cell_steps": offered, "served_fraction_of_offered": stats.executed_cell_steps / offered},
        "latency": {"p50_s": p["p50_s"], "p99_s": p["p99_s"], "completed": len(done),
                    "failed": len(stats.completed) - len(done), "admitted": stats.admitted,
                    "waiting_at_end": stats.waiting_at_end, "active_at_end": stats.active_at_end,
                    "max_active": stats.max_active, "budget_rejections": stats.rejected_budget,
                    "p99_target_s": args.p99_target, "meets_p99_target": bool(p["p99_s"] <= args.p99_target)},
        "e2e": {"value": stats.executed_cell_steps / wall, "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0, "note": "wall clock of the whole window, admission and set-up included"},
        "gpu_launches": stats.ticks, "clocks": clk,
        "audit_vs_fp64": audit,
    }


def audit_served(reqs, done, fraction: float = 0.01) -> dict:
    """Error of served requests against the plain FP64 GPU path on an audit sample (1 % of the
    completed requests, at least one, evenly spaced by request id): each sampled request is
    solved again with float64 fields and the reference's pressure scheme for the same steps,
    and the final cell velocities are compared (relative L2)."""
    from dataclasses import replace

    import numpy as np

    from foilbench_b200.geometry import NacaFoil
    from foilbench_b200.solver import StableFluidsSolver

    if not done:
        return {"sampled": 0}
    by_id = {r.rid: r for r in reqs}
    ordered = sorted(done, key=lambda c: c.rid)
    k = max(1, int(round(fraction * len(ordered))))
    picks = [ordered[int(i * len(ordered) / k)] for i in range(k)]
    errs = []
    for c in picks:
        sc = by_id[c.rid].scenario
        sc64 = replace(sc, precision="float64", solver_options={**sc.solver_options, "pressure_scheme": "reference"})
        sv = StableFluidsSolver()
        sv.initialize(sc64, NacaFoil(sc64.foil), 0)
        for n in range(c.steps):
            sv.advance(sc64.control_at((n + 1) * sc64.output_dt), sc64.output_dt)
        ref = sv.cell_velocity()
        sv.close()
        errs.append(float(np.linalg.norm(c.velocity.astype(np.float64) - ref) / max(np.linalg.norm(ref), 1e-300)))
    return {"sampled": len(picks), "of_completed": len(ordered), "request_ids": [c.rid for c in picks],
            "steps": [c.steps for c in picks], "velocity_rel_l2_max": max(errs),
            "velocity_rel_l2_median": float(np.median(errs))}


def cpu_worker(workload: str, warm: int, timed: int) -> None:
    """One host process of the reference arm: initialise the CPU port (untimed), run `warm`
    untimed advances, report ready, wait for the parent's go on stdin, then run `timed`
    advances and print their cell-substeps and busy seconds."""
    from oracle.stable_fluids import OracleSolver

    w = WORKLOADS[workload]
    sc = make_scenario(w)
    o = OracleSolver(sc)
    o.initialize()
    k = 0
    for _ in range(warm):
        k += 1
        o.advance(sc.control_at(k * sc.output_dt), sc.output_dt)
    print("READY", flush=True)
    sys.stdin.readline()
    tot, subs = 0.0, 0
    for _ in range(timed):
        k += 1
        t0 = time.perf_counter()
        st = o.advance(sc.control_at(k * sc.output_dt), sc.output_dt)
        tot += time.perf_counter() - t0
        subs += st.substeps
    print(json.dumps({"cell_substeps": w["nx"] * w["ny"] * subs, "seconds": tot, "advances": timed}), flush=True)


def run_reference(args) -> dict | None:
    """The reference arm: the reference algorithm (the numpy CPU port of the reference path)
    on the host cores, for the GPU arm's workload, warm-up and step count. The W warm-up and
    K timed advances are spread over P = min(cores, K) single-threaded processes; each process
    initialises its own solver and runs its warm-up advances before a common start, and the
    timed region is the wall time from that start until the last process has finished its
    timed advances. value = cell-substeps of the K timed advances / that wall time;
    ms_per_step = that wall time / K."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return None
    if args.workload not in WORKLOADS:
        return {"impl": "reference", "unavailable": "the reference has no batched or served path: its runner advances "
                "one solver at a time (PY/benchmark/runner.py:240-273); compare with the single-solve lines"}
    w = WORKLOADS[args.workload]
    cores = os.cpu_count() or 1
    if w["nx"] * w["ny"] > PARTS_LIMIT_CELLS:
        # one CPU advance runs for about an hour: a sample formed from timed parts of a substep
        procs = max(1, min(cores, args.steps))
        cb = cpu_sample_subprocess(args.workload, 1, procs)
        value, wall, steps, warm = cb["value"], cb["advance_seconds"], procs, 0
        sample = (cb.get("sample") or "") + f", in each of {procs} processes"
    else:
        procs = max(1, min(cores, args.steps))
        warm_p = [args.warmup // procs + (p < args.warmup % procs) for p in range(procs)]
        timed_p = [args.steps // procs + (p < args.steps % procs) for p in range(procs)]
        env = dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1", MKL_NUM_THREADS="1",
                   CUDA_VISIBLE_DEVICES="")
        ps = [subprocess.Popen([sys.executable, str(Path(__file__).resolve()), "--cpu-worker", args.workload,
                                "--cpu-warm", str(warm_p[p]), "--cpu-timed", str(timed_p[p])],
                               stdin=subprocess.PIPE, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, env=env)
              for p in range(procs)]
        for p in ps:
            line = p.stdout.readline()
            if line.strip() != "READY":
                raise RuntimeError(f"reference worker failed to start: {line!r} {p.stderr.read()[-2000:]}")
        t0 = time.perf_counter()
        for p in ps:
            p.stdin.write("go\n")
            p.stdin.flush()
        outs = []
        for p in ps:
            out, err = p.communicate(timeout=3600)
            if p.returncode != 0:
                raise RuntimeError(f"reference worker failed: {err[-2000:]}")
            outs.append(json.loads(out.strip().splitlines()[-1]))
        wall = time.perf_counter() - t0
        cs = sum(o["cell_substeps"] for o in outs)
        value, steps, warm = cs / wall, args.steps, args.warmup
        sample = (f"{args.steps} timed advances ({max(timed_p)} per process at most) after {args.warmup} warm-up "
                  f"advances over {procs} single-threaded processes, each from its own initialisation; numpy "
                  "restatement of the reference path (" + ("float32 fields with FP64 CG, as the reference runs "
                                                          "them)" if w["precision"] == "float32" else "float64)"))
    return {
        "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": steps,
        "warmup": warm, "ms_per_step": 1e3 * wall / steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64" if w["precision"] == "float32" else "f64",
        "data": "synthetic scenario (seeded, no dataset)", "impl": "reference",
        "config": {"workload": w["name"], "grid": f"{w['nx']}x{w['ny']}", "parallelism": f"{procs} host processes",
                   "timed_region_s": wall,
                   "note": "ms_per_step = wall time of the timed region / timed advances (whole job)"},
        "cpu_baseline": {"value": value, "unit": "cell-steps/s", "cores": procs, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS) + ["c3", "c4"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline sample")
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain-FP64 comparator and the error window")
    ap.add_argument("--no-tune", action="store_true", help="keep the built-in launch heuristic (no autotuning)")
    ap.add_argument("--error-steps", type=int, default=200, help="error window vs the FP64 path (steps)")
    ap.add_argument("--trace", action="store_true", help="print the per-phase device trace instead of a bench line")
    ap.add_argument("--row-transform", default=None, choices=["auto", "fft", "tensor"],
                    help="row DST of the mixed scheme's preconditioner (default: the library's auto choice)")
    ap.add_argument("--seed", type=int, default=2024, help="scenario seed of the batched and served workloads")
    ap.add_argument("--batch-count", type=int, default=64, help="scenarios per batch (batched, served)")
    ap.add_argument("--rate", type=float, default=200.0, help="served: arrivals per second")
    ap.add_argument("--duration", type=float, default=60.0, help="served: arrival window (s)")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="served: wall-clock window of the run (s)")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="served: HBM budget of the solves (GB)")
    ap.add_argument("--p99-target", type=float, default=60.0, help="served: stated p99 latency target (s)")
    ap.add_argument("--cpu-sample", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--cpu-advances", type=int, default=1, help=argparse.SUPPRESS)
    ap.add_argument("--cpu-worker", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--cpu-warm", type=int, default=0, help=argparse.SUPPRESS)
    ap.add_argument("--cpu-timed", type=int, default=1, help=argparse.SUPPRESS)
    args = ap.parse_args()
    global ROW_TRANSFORM
    ROW_TRANSFORM = args.row_transform
    if args.cpu_worker:
        cpu_worker(args.cpu_worker, args.cpu_warm, args.cpu_timed)
        return
    if args.cpu_sample:
        print(json.dumps(cpu_sample(args.cpu_sample, args.cpu_advances)))
        return
    if args.trace:
        run_trace(args)
        return
    if args.warmup < 3 and args.impl == "b200":
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.impl == "b200" and args.workload in ("c3", "c4"):
        out = run_batched(args) if args.workload == "c3" else run_served(args)
        if out is not None:
            print(json.dumps(out))
        if int(os.environ.get("WORLD_SIZE", "1")) > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    out = run_reference(args) if args.impl == "reference" else run_gpu(args)
    if out is not None:
        print(json.dumps(out))
    if int(os.environ.get("WORLD_SIZE", "1")) > 1 and args.impl == "b200":
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
