"""Build recipe of libcoldplate.so: nvcc for sm_100a, in-tree, static cudart."""
from __future__ import annotations

import os
import subprocess

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG_DIR)          # coldplate-solver_b200/
CSRC = os.path.join(ROOT, "csrc")
OUT = os.path.join(ROOT, "libcoldplate.so")
SOURCES = ["cp_solver.cu", "cp_thermal.cu"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr"]


def _sources_mtime() -> float:
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    inc = os.path.join(os.path.dirname(ROOT), "include")
    files += [os.path.join(inc, f) for f in os.listdir(inc)]
    return max(os.path.getmtime(f) for f in files if os.path.exists(f))


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the CUDA sources into libcoldplate.so (skipped when up to date)."""
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= _sources_mtime():
        return OUT
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *NVCC_FLAGS, *[os.path.join(CSRC, s) for s in SOURCES], "-o", OUT + ".tmp"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force=True, verbose=True))
