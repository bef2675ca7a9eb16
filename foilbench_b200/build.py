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
SOURCES = ["fb_lib.cu", "fb_kern_f64.cu", "fb_kern_f32r.cu", "fb_kern_f32m.cu", "fb_noalloc.cu", "fb_kern_batch.cu"]
DEPS = SOURCES + ["fb_step.cuh", "fb_dst.cuh", "fb_fft.cuh", "fb_device.cuh", "fb_umma.cuh"]
NVCC_FLAGS = [
    "-std=c++17",
    "-O3",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
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
    """Compile every translation unit in parallel (-c), then link the shared library."""
    if not force and not stale():
        return TARGET
    out = HERE / "_build"
    out.mkdir(exist_ok=True)
    procs = []
    for src in SOURCES:
        obj = out / (Path(src).stem + ".o")
        cmd = [nvcc(), *NVCC_FLAGS, "-Xptxas", "-v", "-I", str(INCLUDE), "-c", "-o", str(obj), str(CSRC / src)]
        procs.append((src, obj, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)))
    logs = []
    for src, obj, p in procs:
        so, se = p.communicate()
        logs.append(f"== {src}\n{se}")
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src} ({p.returncode}):\n{so}\n{se}")
    (out / "ptxas_info.txt").write_text("\n".join(logs))
    link = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(TARGET),
            *[str(o) for _, o, _ in procs]]
    res = subprocess.run(link, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    if verbose:
        print("\n".join(logs))
    return TARGET


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.verbose))
