"""Parity at the sizes the benchmark numbers are quoted on (GPU tests).

 * the bandwidth model itself (256 x 256 x 128 cells, 8-cell PML, 64 seeded
   dielectric boxes, 4 ports, 16 probes), a short run through the default
   (autotuned) step kernel, against the FP32 CPU oracle and against the
   reference's own CUDA engine (rfnetwork/core/src/solver.cu) on the same
   packed model: relative L2 <= 1e-5 on the full probe matrix;
 * seeded members of the 64-simulation batch at their real sizes (axes
   32..160, 8-cell PML), stepped inside one batch, against the FP32 oracle:
   relative L2 <= 1e-5 per member;
 * the adjoint workload's check at its stated size: a 32 x 32 x 24 copy of the
   microstrip with a design block of proportional size (12 x 12 x 1 above the
   strip, as 48 x 48 x 4 is on the 128 x 128 x 96 model), 11 frequencies in
   8..12 GHz, checkpoints every 32 steps: the GPU gradient against the FP64
   numpy discrete adjoint, relative L2 <= 1e-4.
"""
import copy

import numpy as np
import pytest

import adjoint_model as am
import kernel_model as km
from helpers import rel_l2, run_oracle
from modelgen import configs
from oracle import ref_cuda
from rfnetwork_b200 import _lib

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _engine_probes(s, kernel=None):
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)
    sim = _lib.Simulation(Nx, Ny, Nz)
    if kernel:
        sim.set_kernel(*kernel)
    sim.set_coefficients(co)
    for p in pr:
        src = bool(p["is_source"])
        sim.add_probe(int(p["field"]), p["idx"], src, p["values"][:Nt] if src else None)
    sim.run(Nt)
    rec = sim.probe_values()
    st = sim.stats()
    sim.close()
    return rec, st


@pytest.fixture(scope="module")
def bandwidth_model():
    return configs.boxes(nt=160)


@pytest.mark.parametrize("kernel", [None, (0, 0, 4, 0), (1, 8, 4, 0)])
def test_bandwidth_model_full_grid_vs_oracle(engine_lib, oracle_lib, bandwidth_model, kernel):
    s = bandwidth_model
    rec, st = _engine_probes(s, kernel)
    _, ora = run_oracle(s)
    assert rec.shape == ora.shape and np.abs(ora).max() > 0
    err = rel_l2(rec, ora)
    print(f"256x256x128, 160 steps, kernel {st['variant']}/{st['tile_y']}/{st['stages']}: "
          f"relative L2 vs FP32 oracle {err:.3e}")
    assert err <= TOL


@pytest.mark.skipif(not ref_cuda.available(), reason="reference CUDA engine not built")
def test_bandwidth_model_full_grid_vs_reference_cuda(engine_lib, bandwidth_model):
    s = bandwidth_model
    rec, _ = _engine_probes(s)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = copy.deepcopy(s).pack_inputs(gpu=True)
    ref_cuda.solver_run_cu(co, pr, [], mem, Nx, Ny, Nz, Nt, 0, 0)
    ref = np.array([p["values"][:Nt] for p in pr])
    assert np.isfinite(ref).all() and np.abs(ref).max() > 0
    err = rel_l2(rec, ref)
    print(f"256x256x128, 160 steps: relative L2 vs the reference CUDA engine {err:.3e}")
    assert err <= TOL


@pytest.mark.parametrize("kernel", [(1, 4, 6, 0), (1, 8, 4, 0)])
def test_batch_members_at_real_sizes_vs_oracle(engine_lib, oracle_lib, kernel):
    nt = 120
    members = [configs.batch_member(3, i, nt=nt) for i in (0, 1, 2, 3)]
    sims = []
    for m in members:
        co, pr, mo, mem, Nx, Ny, Nz, Nt = m.pack_inputs(gpu=True)
        sim = _lib.Simulation(Nx, Ny, Nz)
        sim.set_coefficients(co)
        for p in pr:
            src = bool(p["is_source"])
            sim.add_probe(int(p["field"]), p["idx"], src, p["values"][:Nt] if src else None)
        sims.append(sim)
    batch = _lib.Batch(sims)
    batch.set_kernel(*kernel)
    batch.run(nt)
    for m, sim in zip(members, sims):
        rec = sim.probe_values()
        _, ora = run_oracle(m)
        assert np.abs(ora).max() > 0
        err = rel_l2(rec, ora)
        assert err <= TOL, (m.Nx, m.Ny, m.Nz, err)
    batch.close()
    for sim in sims:
        sim.close()


def test_adjoint_on_the_32x32x24_copy_vs_fp64_numpy_adjoint(engine_lib):
    s = configs.microstrip(n=(32, 32, 24), n_pml=4, nt=1000)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)
    out = len(pr) - 1                                   # an output line-voltage probe
    omega = 2 * np.pi * np.linspace(8e9, 12e9, 11) * float(s.dt)
    box = (10, 22, 10, 22, 12, 13)                      # 12 x 12 x 1 design cells in the air above the strip
    sim = _lib.Simulation(Nx, Ny, Nz)
    sim.set_coefficients(co)
    for p in pr:
        sim.add_probe(p["field"], p["idx"], p["is_source"], p["values"][:Nt] if p["is_source"] else None)
    sim.set_dft([(0, out, 1.0)], omega)
    sim.run_checkpointed(Nt, 32)
    X = sim.dft()
    grad = sim.adjoint(2 * X, box)                      # J = sum |X|^2
    ids, rows = sim.material_table()
    sim.close()
    model = am.Model(ids, rows)
    probes = km.shifted_probes(pr)
    src = np.array([p["values"][:Nt] for p in pr], dtype=np.float64)
    rec, hist = am.forward(model, probes, src, Nt, box)
    J, dJ, Xn = am.dft_objective(rec, out, omega)
    assert rel_l2(X[0], Xn) < 1e-5
    ref = am.adjoint(model, probes, dJ, box, hist)
    assert np.abs(ref).max() > 0
    err = rel_l2(grad, ref)
    print(f"32x32x24 copy, 12x12x1 design, 1000 steps: gradient relative L2 vs FP64 numpy adjoint {err:.3e}")
    assert err <= 1e-4
