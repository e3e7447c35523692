"""Pins the CPU oracle and the engine to the reference's own CUDA engine.

The reference's rfnetwork/core/src/solver.cu runs through a harness built
from the reference sources (oracle/ref_cuda.py). Its probe series are the
reference numbers for a model; the oracle (a restatement of the reference's
CPU engine) and the B200 engine must both match them to a relative L2 of
1e-5. The reference GPU build contracts multiply-adds, so bit equality is not
expected.
"""
from __future__ import annotations

import copy

import numpy as np
import pytest

from oracle import ref_cuda
from modelgen import configs
from helpers import rel_l2, run_engine, run_oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_cuda.available(), reason="reference CUDA engine not built")]

TOL = 1e-5


def _models():
    return {
        "microstrip": configs.microstrip(n=(32, 28, 24), n_pml=4, nt=300),
        "boxes": configs.boxes(n=(48, 40, 36), n_pml=6, n_boxes=6, nt=240, n_ports=2, n_probes=4),
    }


def run_reference_cuda(s):
    s2 = copy.deepcopy(s)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s2.pack_inputs(gpu=True)
    ref_cuda.solver_run_cu(co, pr, [], mem, Nx, Ny, Nz, Nt, 0, 0)
    return np.array([p["values"][:Nt] for p in pr])


@pytest.mark.parametrize("name", ["microstrip", "boxes"])
def test_oracle_matches_reference_cuda(name):
    s = _models()[name]
    ref = run_reference_cuda(s)
    _, ora = run_oracle(s)
    assert np.isfinite(ref).all() and np.abs(ref).max() > 0
    err = rel_l2(ora, ref)
    assert err <= TOL, f"{name}: oracle vs reference CUDA relative L2 {err:.3e}"


@pytest.mark.parametrize("name", ["microstrip", "boxes"])
def test_engine_matches_reference_cuda(name):
    s = _models()[name]
    ref = run_reference_cuda(s)
    _, eng = run_engine(s)
    err = rel_l2(eng, ref)
    assert err <= TOL, f"{name}: engine vs reference CUDA relative L2 {err:.3e}"
    for q in range(ref.shape[0]):
        if np.linalg.norm(ref[q]) > 1e-3 * np.linalg.norm(ref):
            e = rel_l2(eng[q], ref[q])
            assert e <= 10 * TOL, f"{name}: probe {q} relative L2 {e:.3e}"


def test_step_time_against_reference_cuda():
    """The drop-in comparison on the bandwidth model (256x256x128, 8-cell PML,
    64 boxes): device time per step of the reference CUDA engine (its four
    kernels per step, read from a CUPTI kernel trace through torch.profiler)
    against this engine's (CUDA events around its run) on the same packed
    model. Prints both (pytest -s)."""
    import json
    import torch
    from torch.profiler import ProfilerActivity, profile
    nt = 200
    s = configs.boxes(nt=nt)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)
    ref_cuda.solver_run_cu(co, copy.deepcopy(pr), [], mem, Nx, Ny, Nz, nt, 0, 0)  # warm-up
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        ref_cuda.solver_run_cu(co, copy.deepcopy(pr), [], mem, Nx, Ny, Nz, nt, 0, 0)
    per_kernel = {}
    for e in prof.events():
        if "update_kernel" in e.name:
            k = per_kernel.setdefault(e.name, [0, 0.0])
            k[0] += 1
            k[1] += e.time_range.elapsed_us()
    ref_ms = sum(v[1] for v in per_kernel.values()) / nt / 1e3   # kernel durations in us
    assert per_kernel and all(v[0] == nt for v in per_kernel.values()), per_kernel
    from rfnetwork_b200 import _lib
    sim = _lib.Simulation(Nx, Ny, Nz)
    sim.set_coefficients(co)
    for p in pr:
        sim.add_probe(p["field"], p["idx"], p["is_source"], p["values"][:Nt] if p["is_source"] else None)
    sim.run(Nt)
    sim.run(Nt)
    ours_ms = sim.stats()["last_run_ms"] / Nt
    sim.close()
    cells = Nx * Ny * Nz
    print(json.dumps({"model": "boxes 256x256x128, 8-cell PML", "steps": nt,
                      "reference_cuda_kernels_us_per_step": {k: round(v[1] / v[0], 1) for k, v in per_kernel.items()},
                      "reference_cuda_ms_per_step": round(ref_ms, 4),
                      "reference_cuda_mcell_per_s": round(cells / ref_ms / 1e3, 1),
                      "b200_ms_per_step": round(ours_ms, 4), "b200_mcell_per_s": round(cells / ours_ms / 1e3, 1),
                      "speedup": round(ref_ms / ours_ms, 2)}))
    assert ours_ms < ref_ms
