"""Builds ``ntustcfdlab_b200/lib/libntcfd.so`` in-tree for sm_100a.

``python -m ntustcfdlab_b200.build`` compiles the CUDA kernels and the C-ABI
(``csrc/ntcfd.cu``), the host set-up code (``csrc/host_grid.cpp``) and the
PLOT3D file I/O (``csrc/host_io.cpp``) with
nvcc for ``-gencode arch=compute_100a,code=sm_100a``.  nvcc cross-compiles,
so the build needs no GPU.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
OUT = os.path.join(LIB_DIR, "libntcfd.so")
SOURCES = ["ntcfd.cu", "host_grid.cpp", "host_io.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise FileNotFoundError("nvcc not found")


def _newest_input() -> float:
    t = 0.0
    for d in (CSRC, os.path.join(HERE, "..", "include")):
        for f in os.listdir(d):
            t = max(t, os.path.getmtime(os.path.join(d, f)))
    return t


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> str:
    """Compiles libntcfd.so unless it is newer than every source."""
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= _newest_input():
        return OUT
    os.makedirs(LIB_DIR, exist_ok=True)
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared",
           "-Xcompiler", "-fPIC,-ffp-contract=off", "-ccbin", "g++",
           "-cudart", "static", "-o", OUT + ".tmp", *[os.path.join(CSRC, s) for s in SOURCES]]
    if extra:
        cmd[1:1] = extra
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed")
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas" in sys.argv else None)
