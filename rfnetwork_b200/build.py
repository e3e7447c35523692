"""Build the engine library in-tree: rfnetwork_b200/librfn_fdtd.so (sm_100a).

    python -m rfnetwork_b200.build [--force] [--verbose]

nvcc compiles the kernels and the C ABI for sm_100a only and links the CUDA
runtime statically, so the library loads with ctypes on any machine with the
NVIDIA driver (and loads, without running anything, on a machine without one).
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "librfn_fdtd.so"
NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["fdtd_api.cu", "fdtd_compile.cpp"]
HEADERS = ["fdtd_kernels.cuh", "fdtd_step_stream.cuh", "fdtd_adjoint.cuh", "fdtd_adjoint_stream.cuh", "fdtd_nf2ff.cuh", "tma.cuh", "fdtd_compile.h"]


def _stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = [CSRC / f for f in SOURCES + HEADERS] + [ROOT / "include" / "fdtd.h"]
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not _stale():
        return LIB
    cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC,-O3",
           "-I", str(ROOT / "include"), "-o", str(LIB)]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += [str(CSRC / f) for f in SOURCES]
    cmd += ["-lpthread"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{res.stdout}\n{res.stderr}")
    if verbose:
        print(res.stdout + res.stderr)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
