"""CPU oracle for the FDTD time-stepping path -- TEST INFRASTRUCTURE ONLY.

`solver_run` mirrors the reference's CPU entry point ``core_func.solver_run``
(rfnetwork/core/src/core_binding.cpp:350-394, called at
rfnetwork/solver.py:1639-1641): it takes the same coefficient dictionary
(CPU shapes, solver.py:1473-1518 with ``end=-1``), probe list, monitor list,
scratch buffer and sizes, and writes probe and monitor results in place.
The arithmetic runs in ``oracle/fdtd_oracle.cpp``, a restatement of
rfnetwork/core/src/solver.cpp.

Only tests/, the smoke check and bench.py's CPU-baseline leg use this module.
The product path never imports it.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "liboracle.so"

# Key order of the coefficient dictionary built at solver.py:1473-1518.
COEFF_NAMES = (
    "Ca_ex_y", "Ca_ex_z", "Cb_ex_y", "Cb_ex_z",
    "Ca_ey_z", "Ca_ey_x", "Cb_ey_z", "Cb_ey_x",
    "Ca_ez_x", "Ca_ez_y", "Cb_ez_x", "Cb_ez_y",
    "Da_hx_y", "Da_hx_z", "Db_hx_y1", "Db_hx_y2", "Db_hx_z1", "Db_hx_z2",
    "Da_hy_z", "Da_hy_x", "Db_hy_z1", "Db_hy_z2", "Db_hy_x1", "Db_hy_x2",
    "Da_hz_x", "Da_hz_y", "Db_hz_x1", "Db_hz_x2", "Db_hz_y1", "Db_hz_y2",
)

_lib = None


def build(force: bool = False) -> Path:
    """Compile the oracle library with g++ (no FMA contraction, see the .cpp header)."""
    src = _HERE / "fdtd_oracle.cpp"
    if LIB_PATH.exists() and not force and LIB_PATH.stat().st_mtime >= src.stat().st_mtime:
        return LIB_PATH
    import subprocess

    cmd = [
        "g++", "-O3", "-std=c++20", "-march=x86-64-v3", "-ffp-contract=off", "-fPIC", "-shared",
        "-pthread", str(src), "-o", str(LIB_PATH),
    ]
    subprocess.run(cmd, check=True)
    return LIB_PATH


def _load():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        lib = ctypes.CDLL(str(LIB_PATH))
        vp = ctypes.c_void_p
        ip = ctypes.POINTER(ctypes.c_int)
        args = [ctypes.c_int] * 5 + [ctypes.POINTER(vp), ctypes.c_int, ip, ip, ip, ctypes.POINTER(vp),
                                     ctypes.c_int, ip, ip, ip, ip, ip, ctypes.POINTER(vp),
                                     ctypes.POINTER(vp), ctypes.c_char_p, ctypes.c_int]
        for name in ("oracle_run_f32", "oracle_run_f64"):
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int
        _lib = lib
    return _lib


def _cpu_shapes(Nx, Ny, Nz):
    """Expected CPU-path coefficient shapes (solver.cpp:284-346, gpu = 0)."""
    cx = (Nx, Ny - 1, Nz - 1)
    cy = (Nx, Ny, Nz - 1)
    cz = (Nx, Ny - 1, Nz)
    dx = (Nx, Ny, Nz)
    dy = (Nx, Ny + 1, Nz)
    dz = (Nx, Ny, Nz + 1)
    return dict(zip(COEFF_NAMES, [cx] * 4 + [cy] * 4 + [cz] * 4 + [dx] * 6 + [dy] * 6 + [dz] * 6))


def _check_array(arr, name, shape, dtype):
    """Shape / dtype / order checks of get_solver_array (solver.cpp:80-117)."""
    if not isinstance(arr, np.ndarray) or arr.ndim != len(shape):
        raise RuntimeError("Invalid data array. Wrong number of dimensions.")
    if arr.dtype != dtype:
        raise RuntimeError("Invalid data array. Must be float type.")
    if not arr.flags["C_CONTIGUOUS"]:
        raise RuntimeError(f"Invalid data array {name}. Must be row ordered (C-style)")
    for i, (a, b) in enumerate(zip(arr.shape, shape)):
        if a != b:
            raise RuntimeError(f"Invalid data array {name}. Expected shape on axis {i} of {b}")


def solver_run(coefficients, probes, monitors, mem, Nx, Ny, Nz, Nt, n_threads, update_interval,
               precision: str = "f32") -> int:
    """Run the CPU oracle with the reference's ``solver_run`` arguments.

    ``precision`` selects the float32 restatement (identical arithmetic to the
    reference) or the float64 one (same discretisation, FP64 state): for
    ``"f64"`` every coefficient, probe and monitor array must be float64 /
    complex128.
    """
    if not isinstance(coefficients, dict):
        raise TypeError("Expected a coefficients dictionary")
    if not isinstance(monitors, list):
        raise TypeError("Expected a monitors list")
    if not isinstance(probes, list):
        raise TypeError("Expected a probes list")
    fdt = np.float32 if precision == "f32" else np.float64
    cdt = np.complex64 if precision == "f32" else np.complex128
    Nx, Ny, Nz, Nt = int(Nx), int(Ny), int(Nz), int(Nt)

    shapes = _cpu_shapes(Nx, Ny, Nz)
    keep = []
    coeff_ptrs = (ctypes.c_void_p * len(COEFF_NAMES))()
    for i, name in enumerate(COEFF_NAMES):
        arr = coefficients[name]
        _check_array(arr, name, shapes[name], fdt)
        keep.append(arr)
        coeff_ptrs[i] = arr.ctypes.data

    if isinstance(mem, np.ndarray):
        if mem.dtype != np.float32 and precision == "f32":
            raise RuntimeError("Invalid data array. Must be float type.")
        if mem.ndim != 1:
            raise RuntimeError("Invalid memory buffer array. Must be 1 dimension.")

    P = len(probes)
    p_field = np.zeros(max(P, 1), dtype=np.int32)
    p_ijk = np.zeros(max(3 * P, 3), dtype=np.int32)
    p_src = np.zeros(max(P, 1), dtype=np.int32)
    p_vals = (ctypes.c_void_p * max(P, 1))()
    for s, p in enumerate(probes):
        if not isinstance(p, dict):
            raise RuntimeError("Expected a list of probe dictionaries")
        v = p["values"]
        if v.ndim != 1:
            raise RuntimeError("Invalid source array. Wrong number of dimensions.")
        if v.dtype != fdt:
            raise RuntimeError("Invalid data array. Must be float type.")
        if not v.flags["C_CONTIGUOUS"]:
            raise RuntimeError("Invalid source array. Must be row ordered (C-style)")
        if v.shape[0] < Nt:
            raise RuntimeError(f"Invalid data source array shape. Expected shape greater or equal to {Nt}")
        p_field[s] = int(p["field"])
        p_ijk[3 * s: 3 * s + 3] = [int(i) for i in p["idx"]]
        p_src[s] = int(p.get("is_source", 0))
        p_vals[s] = v.ctypes.data

    M = len(monitors)
    m_field = np.zeros(max(M, 1), dtype=np.int32)
    m_axis = np.zeros(max(M, 1), dtype=np.int32)
    m_pos = np.zeros(max(M, 1), dtype=np.int32)
    m_step = np.ones(max(M, 1), dtype=np.int32)
    m_nf = np.zeros(max(M, 1), dtype=np.int32)
    m_vals = (ctypes.c_void_p * max(M, 1))()
    m_phase = (ctypes.c_void_p * max(M, 1))()
    for m, mon in enumerate(monitors):
        m_field[m] = int(mon["field"])
        m_axis[m] = int(mon["axis"])
        m_pos[m] = int(mon["position"])
        m_step[m] = int(mon["n_step"])
        vals = mon["values"]
        if "dtft_phase" in mon:
            if vals.dtype != cdt or mon["dtft_phase"].dtype != cdt:
                raise RuntimeError("Invalid data array. Must be complex float32 type.")
            m_nf[m] = int(mon["n_frequencies"])
            m_phase[m] = mon["dtft_phase"].ctypes.data
        elif vals.dtype != fdt:
            raise RuntimeError("Invalid data array. Must be float type.")
        if not vals.flags["C_CONTIGUOUS"]:
            raise RuntimeError("Invalid data array. Must row ordered (C-style)")
        m_vals[m] = vals.ctypes.data

    err = ctypes.create_string_buffer(512)
    ip = ctypes.POINTER(ctypes.c_int)
    fn = _load().oracle_run_f32 if precision == "f32" else _load().oracle_run_f64
    n_threads = max(1, min(int(n_threads), 20))
    rc = fn(Nx, Ny, Nz, Nt, n_threads, coeff_ptrs, P, p_field.ctypes.data_as(ip),
            p_ijk.ctypes.data_as(ip), p_src.ctypes.data_as(ip), p_vals, M,
            m_field.ctypes.data_as(ip), m_axis.ctypes.data_as(ip), m_pos.ctypes.data_as(ip),
            m_step.ctypes.data_as(ip), m_nf.ctypes.data_as(ip), m_vals, m_phase, err, 512)
    if rc != 0:
        raise RuntimeError(err.value.decode())
    return 0


def default_threads() -> int:
    """Host threads the CPU baseline uses: min(nproc, 20) (MAX_THREADS, solver.h:17)."""
    return max(1, min(os.cpu_count() or 1, 20))
