"""Helpers that read the committed golden fixtures (produced by tests/golden/make_golden.py)."""

import json
from pathlib import Path

import numpy as np

from foilbench_b200.models import scenario_from_dict

GOLDEN = Path(__file__).resolve().parent / "golden"


class Trajectory:
    def __init__(self, name: str):
        self.name = name
        self.data = np.load(GOLDEN / f"traj_{name}.npz")
        self.scenario = scenario_from_dict(json.loads(str(self.data["scenario"])))
        self.evidence = json.loads(str(self.data["evidence"]))
        self.meta = json.loads(str(self.data["meta"]))
        self.diagnostics = json.loads(str(self.data["diagnostics"]))

    @property
    def steps(self) -> int:
        return int(self.meta["steps"])

    @property
    def dt(self) -> float:
        return float(self.meta["dt"])

    def has(self, key: str) -> bool:
        return key in self.data.files

    def __getitem__(self, key: str):
        return self.data[key]


def operators():
    d = np.load(GOLDEN / "operators.npz")
    return d, json.loads(str(d["meta"]))


def masks():
    d = np.load(GOLDEN / "masks.npz")
    meta = json.loads(str(d["meta"]))
    out = []
    for m in meta:
        n = m["resolution"][0] * m["resolution"][1]
        bits = np.unpackbits(d[m["name"]])[:n].astype(bool)
        out.append((m, bits.reshape(m["resolution"][1], m["resolution"][0])))
    return out


def geometry():
    return json.loads((GOLDEN / "geometry.json").read_text())["records"]


TRAJECTORIES = [p.stem[len("traj_"):] for p in sorted(GOLDEN.glob("traj_*.npz"))]
