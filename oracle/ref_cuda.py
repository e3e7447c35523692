"""The reference's own CUDA engine, built from its sources -- TEST INFRASTRUCTURE ONLY.

``build()`` compiles rfnetwork/core/src/solver.cu from the reference checkout
(unmodified, nvcc's default code generation as in the reference's setup.py:
``nvcc -Xcompiler -fPIC -I rfnetwork/core/inc solver.cu``, plus the sm_100a
target) together with ``ref_cuda_harness.cu`` into ``oracle/_ref/libref_cuda.so``.
The library travels with the repository to machines without the checkout.

``solver_run_cu`` takes the arguments of the reference binding
(rfnetwork/core/src/cuda_binding.cpp:20-68): the GPU-shaped coefficient
dictionary, the probe list (values overwritten with the recorded series) and
the monitor list. The harness sets ``is_source`` on every probe, as the
reference does (rfnetwork/core/src/solver.cpp:528 stores the dict lookup).

Used by tests/ to pin the CPU oracle and the engine to the reference's own
numbers; never by the product path.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
OUT_DIR = _HERE / "_ref"
LIB_PATH = OUT_DIR / "libref_cuda.so"
REF_ROOT = Path(os.environ.get("RFN_REFERENCE_ROOT", "/root/reference"))

COEFF_NAMES = (
    "Ca_ex_y", "Ca_ex_z", "Cb_ex_y", "Cb_ex_z",
    "Ca_ey_z", "Ca_ey_x", "Cb_ey_z", "Cb_ey_x",
    "Ca_ez_x", "Ca_ez_y", "Cb_ez_x", "Cb_ez_y",
    "Da_hx_y", "Da_hx_z", "Db_hx_y1", "Db_hx_y2", "Db_hx_z1", "Db_hx_z2",
    "Da_hy_z", "Da_hy_x", "Db_hy_z1", "Db_hy_z2", "Db_hy_x1", "Db_hy_x2",
    "Da_hz_x", "Da_hz_y", "Db_hz_x1", "Db_hz_x2", "Db_hz_y1", "Db_hz_y2",
)

_lib = None


def build(force: bool = False) -> Path | None:
    """Compile the reference CUDA engine when the reference checkout is present."""
    src = REF_ROOT / "rfnetwork" / "core" / "src" / "solver.cu"
    inc = REF_ROOT / "rfnetwork" / "core" / "inc"
    harness = _HERE / "ref_cuda_harness.cu"
    if not src.exists():
        return LIB_PATH if LIB_PATH.exists() else None
    if (LIB_PATH.exists() and not force
            and LIB_PATH.stat().st_mtime > max(src.stat().st_mtime, harness.stat().st_mtime)):
        return LIB_PATH
    OUT_DIR.mkdir(exist_ok=True)
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC", "-shared",
           "-Dprivate=public", "-I", str(inc), str(src), str(harness), "-o", str(LIB_PATH)]
    subprocess.run(cmd, check=True, capture_output=True)
    return LIB_PATH


def available() -> bool:
    return LIB_PATH.exists()


def _load():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} is not built (needs the reference checkout)")
        lib = ctypes.CDLL(str(LIB_PATH))
        ip = ctypes.POINTER(ctypes.c_int)
        vp = ctypes.POINTER(ctypes.c_void_p)
        lib.ref_cuda_run.argtypes = [ctypes.c_int] * 4 + [vp, ctypes.c_int, ip, ip, vp, ctypes.c_int,
                                                           ip, ip, ip, ip, ip, vp, vp, ctypes.c_char_p, ctypes.c_int]
        lib.ref_cuda_run.restype = ctypes.c_int
        _lib = lib
    return _lib


def solver_run_cu(coefficients, probes, monitors, mem, Nx, Ny, Nz, Nt, n_threads=0, update_interval=0) -> int:
    """Run the reference CUDA engine with the reference binding's arguments (GPU shapes)."""
    Nx, Ny, Nz, Nt = int(Nx), int(Ny), int(Nz), int(Nt)
    if not probes:
        # solver.cu:799-802, 974, 1000 launch the probe kernels with (n_probes + 7) / 8 blocks,
        # which is an invalid launch for zero probes
        raise ValueError("the reference CUDA engine needs at least one probe")
    keep = []
    cptr = (ctypes.c_void_p * 30)()
    for i, name in enumerate(COEFF_NAMES):
        a = np.ascontiguousarray(coefficients[name], dtype=np.float32)
        if a.shape != (Nx, Ny, Nz):
            raise ValueError(f"{name}: expected shape {(Nx, Ny, Nz)}, got {a.shape}")
        keep.append(a)
        cptr[i] = a.ctypes.data
    P = len(probes)
    p_field = np.array([int(p["field"]) for p in probes], dtype=np.int32)
    p_ijk = np.array([[int(v) for v in p["idx"]] for p in probes], dtype=np.int32).reshape(-1)
    p_vals = (ctypes.c_void_p * P)()
    for q, p in enumerate(probes):
        v = p["values"]
        if v.dtype != np.float32 or not v.flags["C_CONTIGUOUS"] or v.shape[0] < Nt:
            raise ValueError("probe values must be contiguous float32 of length >= Nt")
        p_vals[q] = v.ctypes.data
    M = len(monitors)
    m_field = np.array([int(m["field"]) for m in monitors] or [0], dtype=np.int32)
    m_axis = np.array([int(m["axis"]) for m in monitors] or [0], dtype=np.int32)
    m_pos = np.array([int(m["position"]) for m in monitors] or [0], dtype=np.int32)
    m_step = np.array([int(m["n_step"]) for m in monitors] or [1], dtype=np.int32)
    m_nf = np.array([int(m.get("n_frequencies", 0)) if "dtft_phase" in m else 0 for m in monitors] or [0],
                    dtype=np.int32)
    m_vals = (ctypes.c_void_p * max(M, 1))()
    m_phase = (ctypes.c_void_p * max(M, 1))()
    for i, m in enumerate(monitors):
        m_vals[i] = m["values"].ctypes.data
        m_phase[i] = m["dtft_phase"].ctypes.data if "dtft_phase" in m else None
    ip = ctypes.POINTER(ctypes.c_int)
    err = ctypes.create_string_buffer(512)
    rc = _load().ref_cuda_run(Nx, Ny, Nz, Nt, cptr, P, p_field.ctypes.data_as(ip), p_ijk.ctypes.data_as(ip),
                              p_vals, M, m_field.ctypes.data_as(ip), m_axis.ctypes.data_as(ip),
                              m_pos.ctypes.data_as(ip), m_step.ctypes.data_as(ip), m_nf.ctypes.data_as(ip),
                              m_vals, m_phase, err, 512)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    return 0
