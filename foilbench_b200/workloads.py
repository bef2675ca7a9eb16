"""Seeded synthetic scenarios of the benchmark configurations (no datasets are involved).

* ``single(...)``: one airfoil solve on the 4 x 2-chord domain [-1, 3] x [-1, 1], freestream
  U = (1, 0), foil pivot at the origin, output interval 0.5 h (CFL 0.5 at U = 1).
* ``batched_mix(seed, count)``: the uneven batched configuration: grids drawn uniformly from
  {256x128, 512x256, 768x384, 1024x512}, NACA 4-digit camber 0-4 %, camber position 2-6
  tenths, thickness 9-18 %, angle of attack uniform in [-5, 20] deg, Reynolds number
  log-uniform in [1e2, 1e4]; float32 fields with the FP64-refined pressure solve.
* ``request_stream(seed, rate, duration)``: the served configuration: Poisson arrivals of
  scenarios drawn like ``batched_mix`` with step counts uniform in [100, 2000].
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .models import ControlKeyframe, DomainSpec, FoilSpec, Scenario

GRID_CHOICES = ((256, 128), (512, 256), (768, 384), (1024, 512))


def single(name: str, nx: int, ny: int, naca: str, angle: float, reynolds: float, *, precision: str = "float32",
           tolerance: float = 1.0e-6, scheme: str | None = None, transport: str = "semi-lagrangian",
           extra: dict | None = None) -> Scenario:
    h = min(4.0 / nx, 2.0 / ny)
    opts = {"stable_advection": transport, "stable_cfl": 0.5, "pressure_tolerance": tolerance}
    if scheme is not None:
        opts["pressure_scheme"] = scheme
    if extra:
        opts.update(extra)
    return Scenario(1, name, DomainSpec(2, ((-1.0, 3.0), (-1.0, 1.0)), (nx, ny)), float(reynolds), (1.0, 0.0),
                    FoilSpec(naca, 1.0, (0.0, 0.0)), (ControlKeyframe(0.0, float(angle)),), 1.0e3, 0.5 * h, precision,
                    0, opts)


def _draw(rng: np.random.Generator, k: int) -> Scenario:
    nx, ny = GRID_CHOICES[int(rng.integers(0, len(GRID_CHOICES)))]
    m = int(rng.integers(0, 5))
    p = int(rng.integers(2, 7))
    tt = int(rng.integers(9, 19))
    naca = f"{m}{p if m else 0}{tt:02d}"
    angle = float(rng.uniform(-5.0, 20.0))
    re = float(10.0 ** rng.uniform(2.0, 4.0))
    return single(f"mix-{k:03d}-{nx}x{ny}-naca{naca}-{angle:+.1f}deg-Re{re:.0f}", nx, ny, naca, angle, re)


def batched_mix(seed: int = 2024, count: int = 64) -> list[Scenario]:
    rng = np.random.default_rng(seed)
    return [_draw(rng, k) for k in range(count)]


@dataclass(frozen=True)
class Request:
    rid: int
    arrival_s: float
    steps: int
    scenario: Scenario


def request_stream(seed: int = 7, rate_per_s: float = 200.0, duration_s: float = 60.0, *,
                   min_steps: int = 100, max_steps: int = 2000) -> list[Request]:
    rng = np.random.default_rng(seed)
    out: list[Request] = []
    t = 0.0
    k = 0
    while True:
        t += float(rng.exponential(1.0 / rate_per_s))
        if t > duration_s:
            break
        steps = int(rng.integers(min_steps, max_steps + 1))
        out.append(Request(k, t, steps, _draw(rng, k)))
        k += 1
    return out
