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
