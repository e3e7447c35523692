"""The CPU oracle: determinism, precision behaviour and the reference's error paths."""
import copy

import numpy as np
import pytest

import make_setup_golden as mg
from helpers import derived_series, rel_l2, run_oracle
from modelgen import geometry as geo
from modelgen import solver as S


@pytest.fixture(scope="module")
def model():
    return mg.build_model(S.FDTD_Solver, geo.Box, geo.Rectangle, geo.Line, mg.grid_edges(),
                          lambda s, e: s.generate_mesh(grid=e))


def test_thread_count_invariance(oracle_lib, model):
    # the x-slab split of solver_run (solver.cpp:550-588) must not change any bit
    _, a = run_oracle(model, n_threads=1)
    s3, b = run_oracle(model, n_threads=3)
    s7, c = run_oracle(model, n_threads=7)
    assert np.array_equal(a, b) and np.array_equal(a, c)
    for k in s3.monitors:
        assert np.array_equal(s3.monitors[k]["values"], s7.monitors[k]["values"])


def test_fp32_close_to_fp64(oracle_lib, model):
    s32, a = run_oracle(model, "f32")
    s64, b = run_oracle(model, "f64")
    assert rel_l2(a, b) < 1e-6
    d32, d64 = derived_series(s32), derived_series(s64)
    for k in d32:
        assert rel_l2(d32[k], d64[k]) < 1e-4, k


def test_sources_drive_fields(oracle_lib, model):
    s, vals = run_oracle(model)
    assert np.abs(vals).max() > 0
    v = s.vi_probe_values("v1")
    assert np.abs(v).max() > 0
    # the phasor monitor accumulated something, the time monitor sampled something
    assert np.abs(s.monitors["mx"]["values"]).max() > 0
    assert np.abs(s.monitors["mz"]["values"]).max() > 0


def test_probe_on_grid_edge_rejected(oracle_lib, model):
    co, pr, mo, mem, Nx, Ny, Nz, Nt = copy.deepcopy(model).pack_inputs(gpu=False, n_threads=2)
    pr.append(dict(values=np.zeros(Nt, np.float32), field=1, idx=[0, 3, 3], is_source=0))
    with pytest.raises(RuntimeError, match="Source cannot be placed on grid edge"):
        oracle_lib.solver_run(co, pr, mo, mem, Nx, Ny, Nz, Nt, 2, 0)


def test_shape_errors(oracle_lib, model):
    co, pr, mo, mem, Nx, Ny, Nz, Nt = copy.deepcopy(model).pack_inputs(gpu=False, n_threads=2)
    bad = dict(co)
    bad["Cb_ex_y"] = np.zeros((Nx, Ny, Nz), np.float32)
    with pytest.raises(RuntimeError, match="Expected shape on axis 1"):
        oracle_lib.solver_run(bad, pr, mo, mem, Nx, Ny, Nz, Nt, 2, 0)
    bad["Cb_ex_y"] = np.zeros((Nx, Ny - 1, Nz - 1), np.float64)
    with pytest.raises(RuntimeError, match="Must be float type"):
        oracle_lib.solver_run(bad, pr, mo, mem, Nx, Ny, Nz, Nt, 2, 0)
    with pytest.raises(RuntimeError, match="greater or equal"):
        oracle_lib.solver_run(co, pr, mo, mem, Nx, Ny, Nz, Nt + 5, 2, 0)
