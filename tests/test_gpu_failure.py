"""Failure paths of the engine, exercised without faulting the GPU.

The reference's engine has no error path on the device (solver.cu:1016-1019
only prints a CUDA error). Here every shared-memory pipeline wait of the step
kernels gives up after a bounded number of polls and the run returns
FDTD_ERR_DEVICE, and an end-of-run sentinel reports a diverged run (NaN or
infinite records or fields) as FDTD_ERR_NONFINITE. The tests make the
failures happen on purpose, on the host side: a test hook keeps one plane's
loads from being issued so that the waits for it expire (with a short poll
limit), and coefficients that amplify every step make a run diverge. After
each failure the same handle runs normally again.
"""
import warnings

import numpy as np
import pytest

from modelgen import configs
from rfnetwork_b200 import _lib, cuda_func
from rfnetwork_b200.solver_constants import COEFF_NAMES

pytestmark = pytest.mark.gpu

FDTD_ERR_DEVICE, FDTD_ERR_NONFINITE = 5, 6


def _model_sim(s, kernel):
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)
    sim = _lib.Simulation(Nx, Ny, Nz)
    # 12-plane z chunks: every block streams at least 14 planes, so each one
    # reaches the withheld plane number
    sim.set_kernel(*kernel)
    sim.set_coefficients(co)
    for p in pr:
        src = bool(p["is_source"])
        sim.add_probe(int(p["field"]), p["idx"], src, p["values"][:Nt] if src else None)
    return sim, Nt


@pytest.mark.parametrize("kernel", [(1, 8, 4, 12), (1, 4, 6, 12)])
@pytest.mark.parametrize("withhold", [0, 5])
def test_expired_wait_reports_device_error_and_the_handle_recovers(engine_lib, withhold, kernel):
    s = configs.microstrip(n=(40, 30, 24), n_pml=4, nt=40)
    sim, nt = _model_sim(s, kernel)
    sim.run(nt)
    ref = sim.probe_values()
    assert np.abs(ref).max() > 0
    # 200 polls of at most ~2 us: each step's waits expire within a few ms
    sim.set_debug(wait_limit=200, withhold_plane=withhold)
    with pytest.raises(_lib.FdtdError) as e:
        sim.run(nt)
    assert e.value.code == FDTD_ERR_DEVICE
    assert "gave up waiting" in str(e.value)
    sim.set_debug()
    sim.run(nt)
    assert np.array_equal(sim.probe_values(), ref)
    sim.close()


def _amplifying_sim(shape, nt, gain):
    """Random coefficients whose decay factors are `gain` (> 1 diverges)."""
    rng = np.random.default_rng(3)
    sim = _lib.Simulation(*shape)
    for name in COEFF_NAMES:
        if name.startswith("Ca") or name.startswith("Da"):
            a = np.full(shape, gain)
        else:
            a = rng.uniform(0.0, 0.1, shape) * rng.choice([-1.0, 1.0], shape)
        sim.set_coefficient(name, a.astype(np.float32))
    t = np.arange(nt, dtype=np.float32)
    nx, ny, nz = shape
    sim.add_probe(2, (nx // 2, ny // 2, nz // 2), True, np.sin(0.3 * t) * np.exp(-((t - 10) / 6) ** 2))
    sim.add_probe(0, (nx // 3, ny // 3, nz // 3))
    return sim


@pytest.mark.parametrize("variant", [0, 1])
def test_diverged_run_reports_nonfinite(engine_lib, variant):
    nt = 400
    sim = _amplifying_sim((24, 20, 18), nt, 1.5)
    sim.set_kernel(variant)
    with pytest.raises(_lib.FdtdError) as e:
        sim.run(nt)
    assert e.value.code == FDTD_ERR_NONFINITE
    assert not np.isfinite(sim.probe_values()).all()
    sim.close()
    # a stable model on a fresh handle of the same engine library runs clean
    ok = _amplifying_sim((24, 20, 18), nt, 0.95)
    ok.set_kernel(variant)
    ok.run(nt)
    assert np.isfinite(ok.probe_values()).all()
    ok.close()


def test_drop_in_call_warns_on_divergence_and_writes_results(engine_lib):
    s = configs.microstrip(n=(32, 28, 24), n_pml=4, nt=300)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)
    co = dict(co)
    for name in COEFF_NAMES:
        if name.startswith("Ca") or name.startswith("Da"):
            co[name] = np.full((Nx, Ny, Nz), 1.5, np.float32)
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        cuda_func.solver_run_cu(co, pr, mo, np.zeros(0, np.float32), Nx, Ny, Nz, Nt, 1, 0)
    assert any(issubclass(x.category, RuntimeWarning) and "diverged" in str(x.message) for x in w)
    assert not np.isfinite(pr[0]["values"][:Nt]).all()
