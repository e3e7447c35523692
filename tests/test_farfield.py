"""Far field: the monitor setup and surface currents against the reference's
own Python (tests/golden/farfield_small.npz, made by make_farfield_golden.py),
and the GPU transform (fdtd_nf2ff) against the numpy restatement of the
reference's C++ transform (oracle/nf2ff.py).

Tolerance of the GPU transform: relative L2 <= 1e-5 against the complex128
oracle (FP32 phases and products, FP64 running sums).
"""
import numpy as np
import pytest

import make_farfield_golden as fg
import make_setup_golden as mg
from helpers import rel_l2
from oracle import nf2ff as nf2ff_oracle
from modelgen import geometry as geo
from modelgen import solver as S

GOLD = np.load(mg.HERE / "farfield_small.npz")


def _model():
    s = fg.build_model(S.FDTD_Solver, geo.Box, geo.Rectangle, lambda s, e: s.generate_mesh(grid=e))
    s.pack_inputs(gpu=True)   # sizes the monitor arrays as solve() would
    for name in s.monitors:
        if name.startswith("ff_"):
            s.monitors[name]["values"] = GOLD[f"mon/{name}"]
    s._solved = True          # monitor data injected instead of a run
    return s


def _golden_args():
    J = [[GOLD[f"J/{a}/{j}"] for j in range(2)] for a in range(3)]
    M = [[GOLD[f"M/{a}/{j}"] for j in range(2)] for a in range(3)]
    r = [[GOLD[f"r/{a}/0"], GOLD[f"r/{a}/1"]] for a in range(3)]
    ds = [GOLD[f"ds/{a}"] for a in range(3)]
    pos = [[float(GOLD[f"pos/{a}/{j}"]) for j in range(2)] for a in range(3)]
    return J, M, r, ds, pos


def _ff_data():
    b, t, p = GOLD["beta"], GOLD["theta"], GOLD["phi"]
    return dict(beta=b, theta=t, phi=p, data=np.zeros((2, len(b), len(t), len(p)), dtype=np.complex64))


def test_monitor_setup_matches_reference():
    s = _model()
    assert np.array_equal(s.farfield["idx"], GOLD["ff_idx"])
    assert np.array_equal(s.farfield["surf_pos"], GOLD["surf_pos_m"])
    assert sorted(n for n in s.monitors if n.startswith("ff_")) == sorted(
        k[4:] for k in GOLD.files if k.startswith("mon/"))


def test_surface_currents_bit_exact():
    J, M, r, ds, pos = _model().farfield_currents()
    gJ, gM, gr, gds, gpos = _golden_args()
    for a in range(3):
        assert np.array_equal(ds[a], gds[a])
        for k in range(2):
            assert np.array_equal(r[a][k], gr[a][k])
        for j in range(2):
            assert pos[a][j] == gpos[a][j]
            assert J[a][j].dtype == np.complex64 and np.array_equal(J[a][j], gJ[a][j]), (a, j)
            assert np.array_equal(M[a][j], gM[a][j]), (a, j)


def test_oracle_single_current_element():
    """One x-directed electric current element at the origin radiates
    E_theta = -j beta eta0 / (4 pi) I dl cos th cos ph, E_phi = j beta eta0 / (4 pi) I dl sin ph."""
    z = np.zeros((3, 1, 1, 1), dtype=np.complex64)
    J = [[z.copy(), z.copy()] for _ in range(3)]
    M = [[z.copy(), z.copy()] for _ in range(3)]
    J[2][0][0, 0, 0, 0] = 1.0
    r = [[np.zeros((1, 1), np.float32)] * 2 for _ in range(3)]
    ds = [np.full((1, 1), 1e-6, np.complex64) for _ in range(3)]
    pos = [[0.0, 0.0] for _ in range(3)]
    ff = dict(beta=np.array([200.0], np.float32), theta=np.deg2rad(np.array([30.0, 90.0], np.float32)),
              phi=np.deg2rad(np.array([0.0, 45.0], np.float32)), data=np.zeros((2, 1, 2, 2), np.complex64))
    nf2ff_oracle.nf2ff(J, M, r, ds, pos, ff)
    th, ph = np.deg2rad([30.0, 90.0])[:, None], np.deg2rad([0.0, 45.0])[None, :]
    k = 200.0 * nf2ff_oracle.ETA0 / (4 * np.pi) * 1e-6
    assert np.allclose(ff["data"][0, 0], -1j * k * np.cos(th) * np.cos(ph), rtol=1e-5)
    assert np.allclose(ff["data"][1, 0], 1j * k * np.sin(ph) * np.ones_like(th), rtol=1e-5)


@pytest.mark.gpu
def test_gpu_transform_matches_oracle(engine_lib):
    from rfnetwork_b200 import _lib
    args = _golden_args()
    ref, gpu = _ff_data(), _ff_data()
    nf2ff_oracle.nf2ff(*args, ref)
    _lib.nf2ff(*args, gpu)
    assert np.abs(ref["data"]).max() > 0
    assert rel_l2(gpu["data"], ref["data"]) <= 1e-5, rel_l2(gpu["data"], ref["data"])


@pytest.mark.gpu
def test_gpu_farfield_of_a_run(engine_lib):
    """End to end: the dipole model solved on the engine, then get_farfield_rE
    (currents from the engine's phasor monitors, transform on the GPU) against
    the oracle transform of the same currents."""
    s = fg.build_model(S.FDTD_Solver, geo.Box, geo.Rectangle, lambda s, e: s.generate_mesh(grid=e))
    s.solve(show_progress=False)
    rE = s.get_farfield_rE(fg.THETA, fg.PHI)
    ff = dict(beta=np.array(2 * np.pi * fg.FREQ / S.c0, np.float32), theta=np.deg2rad(fg.THETA).astype(np.float32),
              phi=np.deg2rad(fg.PHI).astype(np.float32), data=np.zeros_like(rE))
    nf2ff_oracle.nf2ff(*s.farfield_currents(), ff)
    assert np.abs(rE).max() > 0
    assert rel_l2(rE, ff["data"]) <= 1e-5


def test_farfield_gain_matches_reference():
    """get_farfield_gain on a seeded far field against the reference's own
    get_farfield_gain (rfnetwork/solver.py:2804-2868) of the same field
    (tests/golden/farfield_gain.npz): projections, port-source DTFT, 4 pi U / P_in."""
    g = np.load(mg.HERE / "farfield_gain.npz")
    s = _model()
    s.get_farfield_rE = lambda theta, phi: g["rE"]
    gain = s.get_farfield_gain(fg.THETA, fg.PHI, polarization=fg.GAIN_POLS)
    assert gain.shape == g["gain"].shape
    np.testing.assert_allclose(gain, g["gain"], rtol=1e-12, atol=0)
    default = s.get_farfield_gain(fg.THETA, fg.PHI)
    np.testing.assert_allclose(default, g["gain"][:2], rtol=1e-12, atol=0)


def test_total_monitor_data():
    """The three components of an e_total monitor brought to common points
    (rfnetwork/solver.py:2750-2802): in-plane components averaged along
    themselves, plane-edge samples dropped, ordered x, y, z."""
    s = mg.build_model(S.FDTD_Solver, geo.Box, geo.Rectangle, geo.Line, mg.grid_edges(),
                       lambda m, e: m.generate_mesh(grid=e))
    for axis, index in (("z", 2), ("x", 5)):
        s.add_field_monitor(f"et{axis}", "e_total", axis, index=index, n_step=2)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)
    rng = np.random.default_rng(7)
    for m in mo:   # seeded samples in place of a run
        m["values"][...] = rng.standard_normal(m["values"].shape).astype(m["values"].dtype)
    s.unpack_results(pr, mo, gpu=True, Nt=Nt)
    s._solved = True
    ex, ey, ez = [s.monitors[f"etz_{a}"]["values"] for a in "xyz"]
    vals, coords = s.get_total_monitor_data("etz")
    assert np.array_equal(vals[0], (ex[:, 1:, 1:-1] + ex[:, :-1, 1:-1]) / 2)
    assert np.array_equal(vals[1], (ey[:, 1:-1, 1:] + ey[:, 1:-1, :-1]) / 2)
    assert np.array_equal(vals[2], ez[:, 1:-1, 1:-1])
    assert coords["component"] == ("x", "y", "z") and len(coords["x"]) == vals.shape[2]
    ex, ey, ez = [s.monitors[f"etx_{a}"]["values"] for a in "xyz"]
    vals, _ = s.get_total_monitor_data("etx")   # plane y-z: y, z in the plane, x normal
    assert np.array_equal(vals[1], (ey[:, 1:, 1:-1] + ey[:, :-1, 1:-1]) / 2)
    assert np.array_equal(vals[2], (ez[:, 1:-1, 1:] + ez[:, 1:-1, :-1]) / 2)
    assert np.array_equal(vals[0], ex[:, 1:-1, 1:-1])
    with pytest.raises(ValueError):
        s.get_total_monitor_data("mz")


def test_dtft_matches_reference():
    """dtft against the reference's utils.dtft (rfnetwork/utils.py:14-71) of a
    seeded series (tests/golden/dtft_small.npz): the direct sum, and the
    low-passed, decimated form of downsample=True."""
    g = np.load(mg.HERE / "dtft_small.npz")
    np.testing.assert_allclose(S.dtft(g["x"], g["f"], float(g["fs"])), g["X"], rtol=1e-12, atol=0)
    np.testing.assert_allclose(S.dtft(g["x"], g["f"], float(g["fs"]), downsample=True), g["X_ds"], rtol=1e-12, atol=0)
