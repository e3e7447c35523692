"""The setup API reproduces the reference's own setup code bit for bit.

tests/golden/setup_small.npz (uniform grid), setup_graded.npz (non-uniform
grid) and setup_edge.npz (uniform grid with PEC edge corrections) hold what rfnetwork/solver.py's solve() passed to the engine
(coefficient dicts for both packings, probe and monitor lists, port records)
for the model in make_setup_golden.build_model, generated by running the
reference's Python code (see make_setup_golden.py).
"""
import numpy as np
import pytest

import make_setup_golden as mg
from modelgen import geometry as geo
from modelgen import solver as S


@pytest.fixture(scope="module", params=sorted(mg.FIXTURES))
def case(request):
    gold = np.load(mg.HERE / request.param)
    model = mg.build_model(S.FDTD_Solver, geo.Box, geo.Rectangle, geo.Line, mg.FIXTURES[request.param](),
                           lambda s, e: s.generate_mesh(grid=e))
    mg.POST_BUILD.get(request.param, lambda m: m)(model)
    return model, gold


@pytest.fixture(scope="module")
def model(case):
    return case[0]


@pytest.fixture(scope="module")
def GOLD(case):
    return case[1]


def test_time_step(model, GOLD):
    assert np.float32(model.dt) == GOLD["dt"]


@pytest.mark.parametrize("kind", ["cpu", "gpu"])
def test_coefficients_bit_exact(model, GOLD, kind):
    co, pr, mo, mem, Nx, Ny, Nz, Nt = model.pack_inputs(gpu=(kind == "gpu"), n_threads=2)
    assert (Nx, Ny, Nz, Nt) == tuple(GOLD["N"])
    for k, v in co.items():
        ref = GOLD[f"{kind}/coef/{k}"]
        assert v.shape == ref.shape, k
        assert v.dtype == np.float32
        assert np.array_equal(v.view(np.uint32), ref.view(np.uint32)), k


@pytest.mark.parametrize("kind", ["cpu", "gpu"])
def test_probes_and_monitors(model, GOLD, kind):
    co, pr, mo, mem, Nx, Ny, Nz, Nt = model.pack_inputs(gpu=(kind == "gpu"), n_threads=2)
    n_ref = len([k for k in GOLD.files if k.startswith(f"{kind}/probe/") and k.endswith("/meta")])
    assert len(pr) == n_ref
    for i, p in enumerate(pr):
        assert np.array_equal(p["values"], GOLD[f"{kind}/probe/{i}/values"])
        assert np.array_equal([p["field"], *p["idx"], p["is_source"]], GOLD[f"{kind}/probe/{i}/meta"])
    for i, m in enumerate(mo):
        assert np.array_equal([m["axis"], m["position"], m["field"], m["n_step"]], GOLD[f"{kind}/monitor/{i}/meta"])
        assert np.array_equal(m["values"].shape, GOLD[f"{kind}/monitor/{i}/shape"])
        if "dtft_phase" in m:
            assert np.array_equal(m["dtft_phase"], GOLD[f"{kind}/monitor/{i}/dtft_phase"])
    if kind == "cpu":
        assert mem.size == int(GOLD["cpu/mem_size"])


def test_ports_and_probe_widths(model, GOLD):
    for i, p in enumerate(model.ports):
        assert np.array_equal(np.asarray(p["Vs_a"]), GOLD[f"port/{i}/Vs_a"])
        assert np.array_equal([p["axis"], p["r0"], p["direction"]], GOLD[f"port/{i}/meta"])
    assert list(model.probes.keys()) == list(GOLD["probe_names"])
    assert np.array_equal(np.array([p["d"] for p in model.probes.values()], dtype=np.float64), GOLD["probe_d"])


def test_errors_mirror_reference():
    s = S.FDTD_Solver(geo.Box(bounds=(0, 0.1, 0, 0.1, 0, 0.1)))
    with pytest.raises(ValueError):
        s.assign_PML_boundaries("w+")
    with pytest.raises(RuntimeError):
        s.pack_inputs()
    s.generate_mesh(grid=mg.grid_edges())
    with pytest.raises(ValueError, match="No port excitations"):
        s.pack_inputs()
