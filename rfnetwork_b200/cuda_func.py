"""Drop-in replacement for the reference's ``rfnetwork.core.cuda_func`` module.

``solver_run_cu`` keeps the exact signature and in-place semantics of the
reference entry point (rfnetwork/core/src/cuda_binding.cpp:20-68, called at
rfnetwork/solver.py:1637-1641): the coefficient dict holds (Nx, Ny, Nz)
float32 arrays, each probe dict's ``values`` array is read as the soft-source
amplitude and overwritten with the recorded field series, and monitor
``values`` arrays are filled in place. The time loop runs in
librfn_fdtd.so on the GPU.

Differences from the reference, all on inputs the reference mishandles:
errors raise ``TypeError`` / ``RuntimeError`` instead of aborting the
process; a probe outside the grid is rejected instead of writing out of
bounds; ``is_source`` is honoured as a flag (the reference tests only that the
key exists, rfnetwork/core/src/solver.cpp:528, which makes no difference for
the zero-valued non-source probes that ``solve()`` builds); each phasor
monitor uses its own ``dtft_phase`` table (the reference GPU path reuses the
last monitor's, solver.cu:842-878). A run that diverges writes its (NaN or
infinite) results in place as the reference does, and also emits a
``RuntimeWarning`` (the engine's end-of-run sentinel, FDTD_ERR_NONFINITE).
"""
from __future__ import annotations

import warnings

import numpy as np

from ._lib import FdtdError, Simulation
from .solver_constants import COEFF_NAMES

_last_info = {}


def last_run_info() -> dict:
    """Statistics of the most recent ``solver_run_cu`` call (rows, split cells, device ms, ...)."""
    return dict(_last_info)


def _check_coefficient(arr, name, shape):
    if not isinstance(arr, np.ndarray) or arr.ndim != 3:
        raise RuntimeError("Invalid data array. Wrong number of dimensions.")
    if arr.dtype != np.float32:
        raise RuntimeError("Invalid data array. Must be float type.")
    if not arr.flags["C_CONTIGUOUS"]:
        raise RuntimeError(f"Invalid data array {name}. Must be row ordered (C-style)")
    for i, (a, b) in enumerate(zip(arr.shape, shape)):
        if a != b:
            raise RuntimeError(f"Invalid data array {name}. Expected shape on axis {i} of {b}")


def solver_run_cu(coefficients, probes, monitors, mem, Nx, Ny, Nz, Nt, n_threads, update_interval) -> int:
    """Run ``Nt`` FDTD steps on the GPU with the reference's ``solver_run_cu`` arguments."""
    if not isinstance(coefficients, dict):
        raise TypeError("Expected a coefficients dictionary")
    if not isinstance(monitors, list):
        raise TypeError("Expected a monitors list")
    if not isinstance(probes, list):
        raise TypeError("Expected a probes list")
    Nx, Ny, Nz, Nt = int(Nx), int(Ny), int(Nz), int(Nt)
    shape = (Nx, Ny, Nz)
    for name in COEFF_NAMES:
        if name not in coefficients:
            raise RuntimeError(f"Missing coefficient array {name}")
        _check_coefficient(coefficients[name], name, shape)
    for p in probes:
        if not isinstance(p, dict):
            raise RuntimeError("Expected a list of probe dictionaries")
        v = p["values"]
        if not isinstance(v, np.ndarray) or v.ndim != 1:
            raise RuntimeError("Invalid source array. Wrong number of dimensions.")
        if v.dtype != np.float32:
            raise RuntimeError("Invalid data array. Must be float type.")
        if not v.flags["C_CONTIGUOUS"]:
            raise RuntimeError("Invalid source array. Must be row ordered (C-style)")
        if v.shape[0] < Nt:
            raise RuntimeError(f"Invalid data source array shape. Expected shape greater or equal to {Nt}")

    _run(coefficients, probes, monitors, Nx, Ny, Nz, Nt)
    return 0


def solver_run_dft(coefficients, probes, monitors, Nx, Ny, Nz, Nt, terms, omega) -> np.ndarray:
    """``solver_run_cu`` plus an FP64 running DFT of probe combinations.

    terms: (series, probe index, weight) triples; omega: radians per step.
    Returns the complex128 array X[series, frequency]. Probe and monitor
    results are written in place as in ``solver_run_cu``.
    """
    if not isinstance(coefficients, dict) or not isinstance(probes, list) or not isinstance(monitors, list):
        raise TypeError("Expected a coefficients dictionary, a probes list and a monitors list")
    return _run(coefficients, probes, monitors, int(Nx), int(Ny), int(Nz), int(Nt), terms, omega)


def _run(coefficients, probes, monitors, Nx, Ny, Nz, Nt, terms=None, omega=None):
    sim = Simulation(Nx, Ny, Nz)
    X = None
    try:
        for name in COEFF_NAMES:
            # borrowed, as the reference's engine borrows the numpy arrays (solver.cpp:80-117);
            # they outlive the simulation, which is closed before this call returns
            sim.set_coefficient(name, coefficients[name], borrow=True)
        for p in probes:
            src = bool(int(p.get("is_source", 0)))
            sim.add_probe(int(p["field"]), p["idx"], src, p["values"][:Nt] if src else None)
        for m in monitors:
            if "dtft_phase" in m:
                sim.add_monitor(int(m["field"]), int(m["axis"]), int(m["position"]), int(m["n_step"]),
                                phase=m["dtft_phase"])
            else:
                sim.add_monitor(int(m["field"]), int(m["axis"]), int(m["position"]), int(m["n_step"]))
        if terms is not None:
            sim.set_dft(terms, omega)
        try:
            sim.run(Nt)
        except FdtdError as e:
            if e.code != 6:  # FDTD_ERR_NONFINITE: the results are complete, only not finite
                raise
            warnings.warn(f"FDTD run diverged: {e}", RuntimeWarning, stacklevel=3)
        if probes:
            rec = sim.probe_values()
            for p, r in zip(probes, rec):
                p["values"][:Nt] = r
        for i, m in enumerate(monitors):
            out = sim.monitor(i)
            vals = m["values"]
            if vals.shape != out.shape:
                raise RuntimeError(f"Monitor {i} values array has shape {vals.shape}, expected {out.shape}")
            vals[...] = out
        if terms is not None:
            X = sim.dft()
        _last_info.clear()
        _last_info.update(sim.stats())
    finally:
        sim.close()
    return X
