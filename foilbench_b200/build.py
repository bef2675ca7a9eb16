"""Build libfoilb200.so in-tree for sm_100a with nvcc.

    python -m foilbench_b200.build [--force]
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
TARGET = HERE / "libfoilb200.so"
SOURCES = ["fb_lib.cu"]
DEPS = ["fb_lib.cu", "fb_step.cuh", "fb_dst.cuh", "fb_device.cuh"]
NVCC_FLAGS = [
    "-std=c++17",
    "-O3",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-Xptxas", "-v",
    "-shared",
    "-Xcompiler", "-fPIC",
    "-Xcompiler", "-O2",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def stale() -> bool:
    if not TARGET.exists():
        return True
    t = TARGET.stat().st_mtime
    deps = [CSRC / n for n in DEPS] + [INCLUDE / "foilb200.h"]
    return any(p.stat().st_mtime > t for p in deps if p.exists())


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not stale():
        return TARGET
    cmd = [nvcc(), *NVCC_FLAGS, "-I", str(INCLUDE), "-o", str(TARGET), *[str(CSRC / s) for s in SOURCES]]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed ({res.returncode}):\n{res.stdout}\n{res.stderr}")
    if verbose:
        print(res.stderr)
    (HERE / "_build").mkdir(exist_ok=True)
    (HERE / "_build" / "ptxas_info.txt").write_text(res.stderr)
    return TARGET


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
