"""The GPU discrete adjoint (fdtd_run_checkpointed + fdtd_adjoint) against the
FP64 numpy discrete adjoint of tests/adjoint_model.py, itself checked against
central finite differences in tests/test_adjoint_model.py.

Tolerance: relative L2 <= 1e-4 over all gradient entries (FP32 fields and
adjoint fields on the GPU, FP64 accumulators; FP64 throughout in numpy).
"""
import numpy as np
import pytest

import adjoint_model as am
import kernel_model as km
from helpers import rel_l2
from rfnetwork_b200 import _lib, configs

pytestmark = pytest.mark.gpu

OMEGA = np.array([0.05, 0.09, 0.13])
BOX = (7, 10, 6, 9, 4, 6)


def _sim(s, variant, every):
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)
    sim = _lib.Simulation(Nx, Ny, Nz)
    sim.set_kernel(variant)
    sim.set_coefficients(co)
    for p in pr:
        sim.add_probe(p["field"], p["idx"], p["is_source"], p["values"][:Nt] if p["is_source"] else None)
    out = len(pr) - 1
    sim.set_dft([(0, out, 1.0)], OMEGA)
    sim.run_checkpointed(Nt, every)
    return sim, pr, Nt, out


@pytest.mark.parametrize("variant,every", [(1, 64), (0, 100), (1, 700)])
def test_gpu_adjoint_matches_numpy_adjoint(engine_lib, variant, every):
    s = configs.microstrip(n=(18, 16, 14), n_pml=3, nt=700)
    sim, pr, nt, out = _sim(s, variant, every)
    X = sim.dft()
    grad = sim.adjoint(2 * X, BOX)          # J = sum |X|^2, dJ/dRe X + i dJ/dIm X = 2 X
    ids, rows = sim.material_table()
    sim.close()
    model = am.Model(ids, rows)
    probes = km.shifted_probes(pr)
    src = np.array([p["values"][:nt] for p in pr], dtype=np.float64)
    rec, hist = am.forward(model, probes, src, nt, BOX)
    J, dJ, Xn = am.dft_objective(rec, out, OMEGA)
    assert rel_l2(X[0], Xn) < 1e-5
    ref = am.adjoint(model, probes, dJ, BOX, hist)
    assert np.abs(ref).max() > 0
    assert rel_l2(grad, ref) <= 1e-4, rel_l2(grad, ref)
