"""Build the sm_100a shared library ``libhitb200.so`` in-tree with nvcc.

    python -m hit_solver_b200.build        # or hit_solver_b200.build.build()

The library is a plain C ABI (include/hitb200.h); it links only the CUDA
runtime.  Builds are incremental on the source timestamps.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libhitb200.so"
SOURCES = ["api.cu"]
HEADERS = ["common.cuh", "reduce.cuh", "weno.cuh", "kernels_reduce.cuh", "kernels_stencil.cuh",
           "kernels_spectra.cuh", "kernels_init.cuh", "sensor_step.cuh",
           "kernels_fft.cuh", "kernels_npnoise.cuh", "ziggurat_table.inc", "stage_persist.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the CUDA 12.9 toolkit is required to build libhitb200.so")


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / s for s in SOURCES + HEADERS] + [ROOT / "include" / "hitb200.h"]
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build():
        return LIB
    cmd = [nvcc_path(), *ARCH, "-O3", "-lineinfo", "-std=c++17",
           "-Xcompiler", "-fPIC", "-shared", "-o", str(LIB.with_suffix(".so.tmp")),
           *[str(CSRC / s) for s in SOURCES], "-cudart", "static"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(LIB.with_suffix(".so.tmp"), LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
