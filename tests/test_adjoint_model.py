"""The FP64 numpy discrete adjoint against central finite differences.

The adjoint model (tests/adjoint_model.py) is the reference the GPU adjoint is
held to; here it is itself checked, on a small PML-bounded microstrip, by
perturbing single E-update coefficients of design-box cells.
"""
import numpy as np
import pytest

import adjoint_model as am
import kernel_model as km
from modelgen import configs
from rfnetwork_b200 import _lib


def _setup():
    s = configs.microstrip(n=(18, 16, 14), n_pml=3, nt=700)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)
    sim = _lib.Simulation(Nx, Ny, Nz)
    sim.set_coefficients(co)
    probes = km.shifted_probes(pr)
    for p in pr:
        sim.add_probe(p["field"], p["idx"], p["is_source"], p["values"] if p["is_source"] else None)
    ids, rows = sim.material_table()
    sim.close()
    src = np.array([p["values"][:Nt] for p in pr], dtype=np.float64)
    return am.Model(ids, rows), probes, src, Nt


@pytest.mark.parametrize("comp,kind", [(0, 0), (1, 1), (2, 2), (2, 0)])
def test_adjoint_matches_finite_differences(engine_lib, comp, kind):
    model, probes, src, nt = _setup()
    box = (7, 10, 6, 9, 4, 6)
    assert not model.es[box[0]:box[1], box[2]:box[3], box[4]:box[5]].any()
    out = len(probes) - 1
    omega = np.array([0.05, 0.09, 0.13])
    rec, hist = am.forward(model, probes, src, nt, box)
    J, dJ, _ = am.dft_objective(rec, out, omega)
    assert J > 0
    grad = am.adjoint(model, probes, dJ, box, hist)
    slot = 4 * comp + (0, 1, 3)[kind]
    g = grad[comp, kind]
    top = np.argsort(np.abs(g).ravel())[-2:]  # the two cells with the largest sensitivity
    for flat in top:
        i, j, k = np.unravel_index(flat, g.shape)
        cell = (box[0] + i, box[2] + j, box[4] + k)
        base = model.coef[slot][cell]
        scale = np.percentile(np.abs(model.coef[slot]), 90)  # the slot's typical size
        h = 1e-4 * max(abs(base), scale)
        Js = []
        for sgn in (1, -1):
            c = model.coef[slot].copy()
            c[cell] = base + sgn * h
            r, _ = am.forward(model.with_coef(slot, c), probes, src, nt)
            Js.append(am.dft_objective(r, out, omega)[0])
        fd = (Js[0] - Js[1]) / (2 * h)
        ad = grad[comp, kind][cell[0] - box[0], cell[1] - box[2], cell[2] - box[4]]
        assert abs(ad) > 1e-9 * J
        assert abs(fd - ad) <= 1e-5 * abs(ad), (cell, fd, ad)


def _light_cone_replay(model, probes, src, start, n0, n1, box, reach, seed):
    """Segment replay the way the engine runs it: two time buffers, the state
    restored into buffer n0 & 1 only (the other holds unrelated values), and
    step n written only to the cells within reach(n) cells (Chebyshev) of the
    box; the history of step n read from buffer n & 1."""
    rng = np.random.default_rng(seed)
    shape = model.shape
    stale = tuple([rng.standard_normal(shape) for _ in range(k)] for k in (3, 3, 6, 6))
    buf = [None, None]
    buf[n0 & 1], buf[(n0 + 1) & 1] = start, stale
    idx = np.indices(shape)
    gap = np.max([np.maximum(0, np.maximum(box[2 * a] - idx[a], idx[a] - (box[2 * a + 1] - 1)))
                  for a in range(3)], axis=0)
    hist = []
    for n in range(n0, n1):
        hist.append(am.box_history(buf[n & 1], box))
        if n + 1 < n1:
            new = am.step(model, probes, src, n, buf[n & 1])
            m = gap <= reach(n)
            old = buf[(n + 1) & 1]
            buf[(n + 1) & 1] = tuple([np.where(m, a, b) for a, b in zip(na, ob)] for na, ob in zip(new, old))
    return hist


def test_light_cone_replay_rule(engine_lib):
    """The engine's checkpointed adjoint replays step n of a segment [n0, n1)
    only within n1-1-n cells of the box. In the FP64 model that gives the
    full forward's box history exactly, even with unrelated values in the
    other time buffer and outside the reach; one cell less does not (the
    history reads H one cell beyond the box)."""
    s = configs.microstrip(n=(30, 24, 20), n_pml=3, nt=80)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)
    sim = _lib.Simulation(Nx, Ny, Nz)
    sim.set_coefficients(co)
    for p in pr:
        sim.add_probe(p["field"], p["idx"], p["is_source"], p["values"] if p["is_source"] else None)
    ids, rows = sim.material_table()
    sim.close()
    model = am.Model(ids, rows)
    probes = km.shifted_probes(pr)
    src = np.array([p["values"][:Nt] for p in pr], dtype=np.float64)
    box = (12, 17, 9, 13, 8, 10)
    n0, n1 = 40, 60
    states = {n0: None}
    _, full = am.forward(model, probes, src, n1, box, states)
    ref = full[n0:n1]
    assert np.abs(ref[-1][0]).max() > 0 and np.abs(ref[-1][1]).max() > 0
    got = _light_cone_replay(model, probes, src, states[n0], n0, n1, box, lambda n: n1 - 1 - n, 1)
    for (e, d), (e_ref, d_ref) in zip(got, ref):
        assert np.array_equal(e, e_ref) and np.array_equal(d, d_ref)
    short = _light_cone_replay(model, probes, src, states[n0], n0, n1, box, lambda n: n1 - 2 - n, 1)
    assert not all(np.array_equal(d, d_ref) for (_, d), (_, d_ref) in zip(short, ref))
