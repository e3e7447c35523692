"""Parity of the CUDA engine with the CPU oracle (GPU tests).

The engine runs from the GPU packing of a model (reference solve(gpu=True)),
the oracle from the CPU packing of the same model; both are unpacked onto the
model the way the reference's solve() does, so probe series, port series and
monitors are compared in the same coordinates.

Tolerances (written per test):
 * FP32 engine vs FP32 oracle: relative L2 <= 1e-5 on every port voltage /
   current series and named probe series, and on the full probe matrix;
 * FP32 engine vs FP64 oracle: relative L2 <= 1e-4 on port voltages, S
   within 0.01 dB / 0.1 deg where |S| > -40 dB;
 * device FP64 DFT vs numpy DTFT of the recorded series: 1e-9 relative.
"""
import copy
import json

import numpy as np
import pytest

import make_setup_golden as mg
from helpers import derived_series, rel_l2, run_engine, run_oracle
from modelgen import configs
from rfnetwork_b200 import _lib
from modelgen import geometry as geo
from modelgen import solver as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    return mg.build_model(S.FDTD_Solver, geo.Box, geo.Rectangle, geo.Line, mg.grid_edges(),
                          lambda s, e: s.generate_mesh(grid=e))


def _compare_series(a, b, tol):
    da, db = derived_series(a), derived_series(b)
    worst = {k: rel_l2(da[k], db[k]) for k in db}
    bad = {k: v for k, v in worst.items() if not v <= tol}
    assert not bad, f"series above {tol}: {bad}"
    return worst


def test_small_model_probes(engine_lib, oracle_lib, small):
    se, pe = run_engine(small)
    so, po = run_oracle(small)
    assert pe.shape == po.shape
    assert rel_l2(pe, po) <= 1e-5
    _compare_series(se, so, 1e-5)


def test_edge_corrected_model(engine_lib, oracle_lib):
    """The small model with PEC edge corrections on the trace (per-cell H rows
    with Db1 != Db2), whose setup tests/golden/setup_edge.npz pins."""
    edge = mg.with_edge_corrections(mg.build_model(S.FDTD_Solver, geo.Box, geo.Rectangle, geo.Line,
                                                   mg.grid_edges(), lambda s, e: s.generate_mesh(grid=e)))
    se, pe = run_engine(edge)
    so, po = run_oracle(edge)
    assert rel_l2(pe, po) <= 1e-5
    _compare_series(se, so, 1e-5)


def test_graded_grid_model(engine_lib, oracle_lib):
    """The same model on a non-uniform grid (cells of 0.005 to 0.02 in), whose
    setup is pinned to the reference by tests/golden/setup_graded.npz."""
    graded = mg.build_model(S.FDTD_Solver, geo.Box, geo.Rectangle, geo.Line, mg.grid_edges_graded(),
                            lambda s, e: s.generate_mesh(grid=e))
    se, pe = run_engine(graded)
    so, po = run_oracle(graded)
    assert rel_l2(pe, po) <= 1e-5
    _compare_series(se, so, 1e-5)
    for k in so.monitors:
        assert rel_l2(se.monitors[k]["values"], so.monitors[k]["values"]) <= 1e-5, k


def test_small_model_monitors(engine_lib, oracle_lib, small):
    se, _ = run_engine(small)
    so, _ = run_oracle(small)
    for k in so.monitors:
        a, b = se.monitors[k]["values"], so.monitors[k]["values"]
        assert a.shape == b.shape, k
        assert rel_l2(a, b) <= 1e-5, k


def test_batch_equals_single_runs(engine_lib):
    """Three uneven simulations in one batch give the same bits as three single runs."""
    nt = 200
    members = [configs.batch_member(7, i, nt=nt, size_range=(20, 40), n_pml=4) for i in range(3)]
    singles = []
    for m in members:
        _, rec = run_engine(m)
        singles.append(rec)
    sims = []
    for m in members:
        co, pr, mo, mem, Nx, Ny, Nz, Nt = m.pack_inputs(gpu=True)
        sim = _lib.Simulation(Nx, Ny, Nz)
        sim.set_coefficients(co)
        for p in pr:
            sim.add_probe(p["field"], p["idx"], p["is_source"], p["values"] if p["is_source"] else None)
        sims.append(sim)
    batch = _lib.Batch(sims)
    batch.run(nt)
    for sim, ref in zip(sims, singles):
        assert np.array_equal(sim.probe_values(), ref)
    assert batch.stats()["step_launches"] == nt


def test_device_dft_matches_numpy(engine_lib, small):
    f = np.linspace(1e9, 20e9, 21)
    se, _ = run_engine(small, frequency=f)
    S_dev = se.get_sparameters_device()
    S_np = se.get_sparameters(f)
    # the device transforms the FP32 probe series in FP64; numpy first forms the
    # port series in float32 (solver.py:2482-2496) -- agreement to ~1e-6
    assert rel_l2(S_dev, S_np) < 1e-5
    names, X = se.dft["names"], se.dft["X"]
    from modelgen.solver import dtft
    vp, ip = se.port_vi_series(0)
    Xv = dtft(vp.astype(np.float64), f, 1 / se.dt)
    assert rel_l2(X[names.index("V1")], Xv) < 1e-6


def test_microstrip_full_size(engine_lib, oracle_lib):
    """64x64x48, 10-cell PML on six faces, 2000 steps, 101-point S11/S21."""
    s = configs.microstrip()
    f = configs.microstrip_frequencies()
    se, pe = run_engine(s, frequency=f)
    so, po = run_oracle(s, "f32")
    s64, _ = run_oracle(s, "f64")
    assert rel_l2(pe, po) <= 1e-5
    _compare_series(se, so, 1e-5)
    # FP32 engine against the FP64 run of the same discretisation
    for i in range(len(s.ports)):
        assert rel_l2(se.port_vi_series(i)[0], s64.port_vi_series(i)[0]) <= 1e-4
    S32 = se.get_sparameters_device()[:, :, 0]
    S64 = s64.get_sparameters(f)[:, :, 0]
    mag = 20 * np.log10(np.abs(S64))
    keep = mag > -40
    ddb = np.abs(20 * np.log10(np.abs(S32)) - mag)[keep]
    dph = np.abs(np.angle(S32 / S64, deg=True))[keep]
    # the measured errors of this result (pytest -s prints them)
    print(json.dumps({"model": "microstrip 64x64x48, 10-cell PML, 2000 steps",
                      "probes_vs_fp32_oracle_rel_l2": float(rel_l2(pe, po)),
                      "port_v_vs_fp64_rel_l2": [float(rel_l2(se.port_vi_series(i)[0], s64.port_vi_series(i)[0]))
                                                for i in range(len(s.ports))],
                      "s_vs_fp64_max_db": float(ddb.max()), "s_vs_fp64_max_deg": float(dph.max())}))
    assert ddb.max() <= 0.01 and dph.max() <= 0.1, (ddb.max(), dph.max())
    # physical sanity: a matched 50-ohm-ish line transmits most of the power
    assert np.abs(S32[:, 1]).max() > 0.5


def test_no_nan_after_long_run(engine_lib):
    s = configs.boxes(n=(64, 64, 48), n_pml=8, n_boxes=8, nt=600)
    se, pe = run_engine(s)
    assert np.isfinite(pe).all()
    assert np.abs(pe).max() > 0


def _engine_probe_matrix(s, variant, graph=True, **kw):
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)
    sim = _lib.Simulation(Nx, Ny, Nz)
    sim.set_kernel(variant, **kw)
    sim.set_graph(graph)
    sim.set_coefficients(co)
    for p in pr:
        sim.add_probe(p["field"], p["idx"], p["is_source"], p["values"] if p["is_source"] else None)
    sim.run(Nt)
    out = sim.probe_values()
    st = sim.stats()
    sim.close()
    return out, st


@pytest.mark.parametrize("ty,stages,zchunk", [(8, 3, 0), (8, 4, 5), (4, 4, 0), (4, 5, 62), (6, 3, 7), (6, 4, 0),
                                              (12, 3, 0)])
def test_stream_kernel_bitwise_equals_plain(engine_lib, ty, stages, zchunk):
    """The streaming kernel evaluates the same expressions as the plain one,
    on the microstrip (PEC, substrate, ports) and on a lossy box model whose
    ports are soft-source cells outside the PML."""
    models = (configs.microstrip(n=(72, 40, 30), n_pml=5, nt=150),
              configs.boxes(n=(70, 45, 38), n_pml=6, n_boxes=6, nt=120, n_ports=2, n_probes=4))
    for s in models:
        a, sa = _engine_probe_matrix(s, 0)
        b, sb = _engine_probe_matrix(s, 1, tile_y=ty, stages=stages, zchunk=zchunk)
        assert sa["variant"] == 0 and sb["variant"] == 1
        assert np.abs(a).max() > 0
        assert np.array_equal(a, b)


@pytest.mark.parametrize("variant", [0, 1])
def test_host_launched_steps_equal_graph_replay(engine_lib, variant):
    """fdtd_set_graph(0): the same launches issued step by step from the host."""
    s = configs.microstrip(n=(40, 30, 24), n_pml=4, nt=200)
    a, _ = _engine_probe_matrix(s, variant)
    b, sb = _engine_probe_matrix(s, variant, graph=False)
    assert sb["step_launches"] == 200
    assert np.abs(a).max() > 0 and np.array_equal(a, b)


@pytest.mark.parametrize("ty,stages,zchunk", [(8, 6, 0), (4, 6, 4)])
def test_stream_kernel_one_list_equals_plain(engine_lib, monkeypatch, ty, stages, zchunk):
    """Every tile through the general streaming kernel (its interior path for
    the plain tiles, one launch per step): the plain kernel's bits."""
    monkeypatch.setenv("RFN_FDTD_ONE_LIST", "1")
    s = configs.microstrip(n=(72, 40, 30), n_pml=5, nt=150)
    a, sa = _engine_probe_matrix(s, 0)
    b, sb = _engine_probe_matrix(s, 1, tile_y=ty, stages=stages, zchunk=zchunk)
    assert sb["variant"] == 1 and sb["step_launches"] == 150
    assert np.abs(a).max() > 0
    assert np.array_equal(a, b)
