"""The GPU discrete adjoint (fdtd_run_checkpointed or fdtd_run_recorded, then
fdtd_adjoint) against the FP64 numpy discrete adjoint of tests/adjoint_model.py,
itself checked against central finite differences in tests/test_adjoint_model.py.

Tolerance: relative L2 <= 1e-4 over all gradient entries (FP32 fields and
adjoint fields on the GPU, FP64 accumulators; FP64 throughout in numpy).
"""
import numpy as np
import pytest

import adjoint_model as am
import kernel_model as km
from helpers import rel_l2
from modelgen import configs
from rfnetwork_b200 import _lib

pytestmark = pytest.mark.gpu

OMEGA = np.array([0.05, 0.09, 0.13])
BOX = (7, 10, 6, 9, 4, 6)


# output line voltage (E probes), input current (H loop around the strip), and
# the input voltage on the source cells (split E cells)
TERMS = ([(0, p, 1.0) for p in (4, 5, 6, 7)]
         + [(1, p, w) for p, w in zip(range(8, 16), (1.0, -1.0, 1.0, -1.0, 1.0, -1.0, 0.5, -0.5))]
         + [(2, p, -1.0) for p in (0, 1, 2, 3)])


def _make(s, variant, terms=None):
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)
    sim = _lib.Simulation(Nx, Ny, Nz)
    sim.set_kernel(variant)
    sim.set_coefficients(co)
    for p in pr:
        sim.add_probe(p["field"], p["idx"], p["is_source"], p["values"][:Nt] if p["is_source"] else None)
    out = len(pr) - 1
    sim.set_dft(terms or [(0, out, 1.0)], OMEGA)
    return sim, pr, Nt, out


def _sim(s, variant, every, terms=None, box=BOX):
    sim, pr, Nt, out = _make(s, variant, terms)
    if every:
        sim.run_checkpointed(Nt, every)
    else:
        sim.run_recorded(Nt, box)
    return sim, pr, Nt, out


def _series_objective(rec, terms, omega):
    """X_s = sum over the series' terms of w DTFT(rec_p); J = sum |X|^2; dJ/drec."""
    ph = np.exp(-1j * np.outer(omega, np.arange(rec.shape[1])))
    X = np.zeros((max(t[0] for t in terms) + 1, len(omega)), dtype=complex)
    for se, p, w in terms:
        X[se] += w * (ph @ rec[p])
    g = np.zeros_like(rec)
    for se, p, w in terms:
        g[p] += w * 2 * np.real(np.conj(X[se]) @ ph)
    return X, g


@pytest.mark.parametrize("variant,every", [(1, 64), (0, 100), (1, 700), (1, 0), (0, 0)])
def test_gpu_adjoint_matches_numpy_adjoint(engine_lib, variant, every):
    """every = 0: recorded box history instead of checkpoints."""
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


@pytest.mark.parametrize("every", [0, 50])
def test_gpu_adjoint_of_port_series(engine_lib, every):
    """Objective over voltage and current series: adjoint sources at split
    (source) E cells and at H probes."""
    s = configs.microstrip(n=(18, 16, 14), n_pml=3, nt=500)
    sim, pr, nt, _ = _sim(s, 1, every, TERMS)
    X = sim.dft()
    grad = sim.adjoint(2 * X, BOX)
    stats = sim.stats()
    ids, rows = sim.material_table()
    sim.close()
    assert stats["adjoint_launches"] == nt and stats["adjoint_ms"] > 0
    model = am.Model(ids, rows)
    probes = km.shifted_probes(pr)
    src = np.array([p["values"][:nt] for p in pr], dtype=np.float64)
    rec, hist = am.forward(model, probes, src, nt, BOX)
    Xn, dJ = _series_objective(rec, TERMS, OMEGA)
    assert rel_l2(X, Xn) < 1e-5
    ref = am.adjoint(model, probes, dJ, BOX, hist)
    assert rel_l2(grad, ref) <= 1e-4, rel_l2(grad, ref)


def test_gpu_batch_adjoint_equals_single_runs(engine_lib):
    """Batched recorded runs and one batched adjoint sweep give each member's
    single-run gradient bit for bit (same arithmetic per cell)."""
    models = [configs.microstrip(n=(18, 16, 14), n_pml=3, nt=400),
              configs.microstrip(n=(23, 19, 15), n_pml=3, nt=400)]
    boxes = [BOX, (9, 13, 7, 10, 4, 6)]
    single = []
    for s, box in zip(models, boxes):
        sim, _, _, _ = _sim(s, 1, 0, TERMS, box)
        X = sim.dft()
        single.append((X, sim.adjoint(2 * X, box)))
        sim.close()
    sims = [_make(s, 1, TERMS)[0] for s in models]
    b = _lib.Batch(sims)
    b.run_recorded(400, boxes)
    Xs = [sim.dft() for sim in sims]
    grads = b.adjoint([2 * X for X in Xs])
    assert b.stats()["adjoint_launches"] == 400
    b.close()
    for sim in sims:
        sim.close()
    for (X1, g1), X, g in zip(single, Xs, grads):
        assert np.array_equal(X1, X)
        assert np.array_equal(g1, g)


def test_gpu_box_patch_runs_equal_full_arrays(engine_lib):
    """Runs after fdtd_set_box_coefficients (table patched in place, captured
    graph kept) equal runs of a fresh simulation given the patched arrays."""
    from test_box_coefficients import _coefs, _patched
    s = configs.microstrip(n=(18, 16, 14), n_pml=3, nt=300)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)

    def fresh(c):
        sim = _lib.Simulation(Nx, Ny, Nz)
        sim.set_coefficients(c)
        for p in pr:
            sim.add_probe(p["field"], p["idx"], p["is_source"], p["values"][:Nt] if p["is_source"] else None)
        return sim

    sim = fresh(co)
    sim.run(Nt)
    cur = co
    for seed in (1, 2, 3):
        coefs = _coefs(cur, BOX, seed)
        sim.set_box_coefficients(BOX, coefs)
        sim.run(Nt)
        cur = _patched(cur, BOX, coefs)
        ref = fresh(cur)
        ref.run(Nt)
        assert np.array_equal(sim.probe_values(), ref.probe_values())
        ref.close()
    sim.close()



@pytest.mark.parametrize("every,graded", [(0, False), (40, False), (0, True)])
def test_gpu_stream_adjoint_equals_plain_adjoint(engine_lib, every, graded, monkeypatch):
    """The streaming reverse step (RFN_ADJ_STREAM=1, after streaming forward
    runs) gives the plain reverse step's gradient (after plain forward runs)
    bit for bit: same per-cell arithmetic with fixed rounding, on a model of
    several tiles along x, y and z with split tiles, plain tiles and records
    at split cells."""
    s = configs.microstrip(n=(70, 44, 37), n_pml=5, nt=160, graded=graded)
    box = (30, 42, 18, 26, 5, 9)
    # output E probes, H probes around the strip, source (split E) cells
    terms = ([(0, p, 1.0) for p in (20, 21, 22, 23)] + [(1, p, (-1.0) ** p) for p in range(40, 48)]
             + [(2, p, -1.0) for p in (0, 1, 2, 3)])
    out = {}
    for variant in (0, 1):
        monkeypatch.setenv("RFN_ADJ_STREAM", str(variant))
        sim, _, nt, _ = _sim(s, variant, every, terms, box)
        X = sim.dft()
        g = sim.adjoint(2 * X, box)
        assert sim.stats()["adjoint_launches"] == nt
        sim.close()
        out[variant] = (X, g)
    assert np.array_equal(out[0][0], out[1][0])
    assert np.abs(out[0][1]).max() > 0
    assert np.array_equal(out[0][1], out[1][1])


def test_gpu_batch_checkpointed_adjoint_equals_recorded(engine_lib):
    """fdtd_batch_run_checkpointed + fdtd_batch_adjoint (the segments of all
    members replayed together) give the gradients of the recorded batch and
    of single checkpointed runs bit for bit: the replay repeats the forward
    arithmetic exactly."""
    models = [configs.microstrip(n=(18, 16, 14), n_pml=3, nt=400),
              configs.microstrip(n=(23, 19, 15), n_pml=3, nt=400)]
    boxes = [BOX, (9, 13, 7, 10, 4, 6)]
    single = []
    for s, box in zip(models, boxes):
        sim, _, _, _ = _sim(s, 1, 50, TERMS, box)
        X = sim.dft()
        single.append((X, sim.adjoint(2 * X, box)))
        sim.close()
    sims = [_make(s, 1, TERMS)[0] for s in models]
    b = _lib.Batch(sims)
    out = {}
    for mode in ("checkpointed", "recorded"):
        if mode == "checkpointed":
            b.run_checkpointed(400, 50, boxes)
        else:
            b.run_recorded(400, boxes)
        Xs = [sim.dft() for sim in sims]
        out[mode] = (Xs, b.adjoint([2 * X for X in Xs]))
        assert b.stats()["adjoint_launches"] == 400
    b.close()
    for sim in sims:
        sim.close()
    for i, (X1, g1) in enumerate(single):
        for mode in ("checkpointed", "recorded"):
            assert np.array_equal(out[mode][0][i], X1)
            assert np.array_equal(out[mode][1][i], g1)


def test_gpu_light_cone_replay_equals_recorded(engine_lib, monkeypatch):
    """Checkpointed segment replays that run only the tiles within reach of
    the box (reach = the steps left before the segment's last history) give
    the recorded-history gradient bit for bit, as full-grid replays do, and
    leave the forward's probe records as the forward wrote them."""
    s = configs.microstrip(n=(96, 64, 40), n_pml=6, nt=300)
    box = (40, 52, 28, 36, 10, 13)
    grads = {}
    for mode in ("recorded", "cone", "full"):
        if mode == "full":
            monkeypatch.setenv("RFN_REPLAY_FULL", "1")
        sim, pr, nt, _ = _make(s, 1, TERMS)
        sim.set_kernel(1, tile_y=8, stages=6)  # the streaming kernels, whose tile lists the replays cut
        if mode == "recorded":
            sim.run_recorded(nt, box)
        else:
            sim.run_checkpointed(nt, 60)
        rec0 = sim.probe_values()
        X = sim.dft()
        grads[mode] = sim.adjoint(2 * X, box)
        assert np.array_equal(sim.probe_values(), rec0), mode
        sim.close()
    assert np.abs(grads["recorded"]).max() > 0
    assert np.array_equal(grads["cone"], grads["recorded"])
    assert np.array_equal(grads["full"], grads["recorded"])
