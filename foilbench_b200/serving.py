"""Served Stable Fluids solves: a continuous-batching request loop on one GPU.

Requests (a scenario and a number of output steps) arrive over time. The loop admits waiting
requests in arrival order while the device context's HBM budget accepts another solver and the
batch has a free member slot; every tick advances all admitted solves by one output interval
in batched launches (``foilbench_b200.batch``), so requests that arrive while others run join
the next tick and their work shares the launches. A request leaves as soon as its last step is
done; its latency is completion time minus arrival time. The reference has no serving layer;
each solve inside it advances exactly as ``StableFluidsSolver.advance`` would.
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import Callable, Sequence

import numpy as np

from . import _native as N
from .batch import StableFluidsBatch
from .geometry import NacaFoil
from .models import NumericalFailure
from .solver import StableFluidsSolver
from .workloads import Request


@dataclass
class Completed:
    rid: int
    arrival_s: float
    admitted_s: float
    finished_s: float
    steps: int
    cell_steps: int
    failed: str = ""
    velocity: np.ndarray | None = None

    @property
    def latency_s(self) -> float:
        return self.finished_s - self.arrival_s


@dataclass
class _Active:
    req: Request
    solver: StableFluidsSolver
    admitted_s: float
    done_steps: int = 0
    cell_steps: int = 0


@dataclass
class ServeStats:
    completed: list[Completed] = field(default_factory=list)
    ticks: int = 0
    busy_s: float = 0.0
    device_s: float = 0.0
    max_active: int = 0
    rejected_budget: int = 0
    waiting_at_end: int = 0
    active_at_end: int = 0
    admitted: int = 0
    executed_cell_steps: int = 0

    def latency_percentiles(self) -> dict[str, float]:
        lat = np.array([c.latency_s for c in self.completed if not c.failed])
        if lat.size == 0:
            return {"p50_s": float("nan"), "p99_s": float("nan")}
        return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99))}

    @property
    def cell_steps(self) -> int:
        return sum(c.cell_steps for c in self.completed)


class ServedSolves:
    """Request loop over one device context.

    ``hbm_budget``: bytes the solvers may hold (0 = unlimited); ``max_members``: solves per
    batched launch (at most one per SM); ``clock``: seconds since start (wall clock by
    default; tests pass a tick counter); ``keep_fields``: keep each finished request's cell
    velocity (for checks)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0, max_members: int = 64,
                 clock: Callable[[], float] | None = None, keep_fields: bool = False):
        self.ctx = N.Context(device, hbm_budget)
        self.max_members = int(max_members)
        self.keep_fields = keep_fields
        t0 = time.perf_counter()
        self.clock = clock or (lambda: time.perf_counter() - t0)

    def _admit(self, req: Request, now: float) -> _Active | None:
        s = StableFluidsSolver(context=self.ctx)
        try:
            s.initialize(req.scenario, NacaFoil(req.scenario.foil), 0)
        except N.NativeError as err:
            if err.code == N.FB_ERR_BUDGET:
                s.close()
                return None
            raise
        return _Active(req, s, now)

    def run(self, requests: Sequence[Request], *, until_s: float | None = None,
            on_tick: Callable[[int], None] | None = None) -> ServeStats:
        pending = sorted(requests, key=lambda r: r.arrival_s)
        waiting: list[Request] = []
        active: list[_Active] = []
        stats = ServeStats()
        batch: StableFluidsBatch | None = None
        members: tuple[int, ...] = ()
        while pending or waiting or active:
            now = self.clock()
            if until_s is not None and now >= until_s:
                break
            while pending and pending[0].arrival_s <= now:
                waiting.append(pending.pop(0))
            while waiting and len(active) < self.max_members:
                a = self._admit(waiting[0], now)
                if a is None:
                    stats.rejected_budget += 1
                    break
                waiting.pop(0)
                active.append(a)
                stats.admitted += 1
            if not active:
                if pending:
                    wait = pending[0].arrival_s - self.clock()
                    if wait > 0:
                        time.sleep(min(wait, 0.05))
                continue
            stats.max_active = max(stats.max_active, len(active))
            ids = tuple(a.req.rid for a in active)
            if ids != members:
                if batch is not None:
                    batch.close()
                batch = StableFluidsBatch([a.solver for a in active])
                members = ids
            t0 = time.perf_counter()
            controls, dts = [], []
            for a in active:
                sc = a.req.scenario
                controls.append(sc.control_at((a.done_steps + 1) * sc.output_dt))
                dts.append(sc.output_dt)
            reps = batch.advance(controls, dts)
            stats.busy_s += time.perf_counter() - t0
            stats.ticks += 1
            dev_ms = 0.0
            still: list[_Active] = []
            for a, r in zip(active, reps):
                cells = a.req.scenario.domain.nx * a.req.scenario.domain.ny
                if isinstance(r, NumericalFailure):
                    self._finish(a, stats, self.clock(), failed=f"{r.reason}: {r}")
                    continue
                dev_ms = r.evidence["device_ms"]
                a.done_steps += 1
                a.cell_steps += cells * r.substeps
                stats.executed_cell_steps += cells * r.substeps
                if a.done_steps >= a.req.steps:
                    self._finish(a, stats, self.clock())
                else:
                    still.append(a)
            stats.device_s += dev_ms / 1e3
            active = still
            if on_tick is not None:
                on_tick(stats.ticks)
        if batch is not None:
            batch.close()
        stats.waiting_at_end = len(waiting) + len(pending)
        stats.active_at_end = len(active)
        for a in active:
            a.solver.close()
        return stats

    def _finish(self, a: _Active, stats: ServeStats, now: float, failed: str = "") -> None:
        vel = a.solver.cell_velocity() if (self.keep_fields and not failed) else None
        stats.completed.append(Completed(a.req.rid, a.req.arrival_s, a.admitted_s, now, a.done_steps, a.cell_steps,
                                         failed, vel))
        a.solver.close()
