"""torch.autograd through the engine: dJ/dtheta of a permittivity design.

J = sum over three frequencies of |DFT of the output line voltage probe|^2;
the design is a 4 x 3 x 2-cell block of the substrate beside the strip, clear
of the PML, the ground plane and the strip, with eps_r = 1 + 9 sigmoid(theta).

The GPU gradient (FP32 fields, FP64 accumulators) is checked against central
finite differences, h = 1e-3 on theta, on 16 seeded voxels, of the same
discretisation run in FP64 (tests/adjoint_model.py on the table the library
compiles for each perturbed design). Finite differences of the FP32 GPU
forward itself would drown in its rounding. Tolerance: 1e-3 of the largest
gradient entry.
"""
import numpy as np
import pytest
import torch

import adjoint_model as am
import kernel_model as km
from modelgen import configs
from rfnetwork_b200 import _lib
from rfnetwork_b200.adjoint import FDTDDesign

pytestmark = pytest.mark.gpu

BOX = (12, 16, 6, 9, 8, 10)  # substrate cells (z 6..9) beside the strip (y 11..16)


def _fp64_objective(design, probes, src, out, omega, eps_r):
    """J of the FP64 model for one design, through the table the library compiles."""
    with torch.no_grad():
        coefs = design.coefficients(eps_r).numpy()
    bx0, bx1, by0, by1, bz0, bz1 = design.box
    co = {k: v.copy() for k, v in design.base.items()}
    names = (("Ca_ex_y", "Ca_ex_z", "Cb_ex_y", "Cb_ex_z"), ("Ca_ey_z", "Ca_ey_x", "Cb_ey_z", "Cb_ey_x"),
             ("Ca_ez_x", "Ca_ez_y", "Cb_ez_x", "Cb_ez_y"))
    for c, (ca1, ca2, cb1, cb2) in enumerate(names):
        for n, k in ((ca1, 0), (ca2, 0), (cb1, 1), (cb2, 2)):
            co[n][bx0:bx1, by0:by1, bz0:bz1] = coefs[c, k].astype(np.float32)
    sim = _lib.Simulation(*design.shape)
    sim.set_coefficients(co)
    for p in design.probes:
        sim.add_probe(p["field"], p["idx"], p["is_source"], p["values"][:design.nt] if p["is_source"] else None)
    ids, rows = sim.material_table()
    sim.close()
    rec, _ = am.forward(am.Model(ids, rows), probes, src, design.nt)
    return am.dft_objective(rec, out, omega)[0]


def test_design_gradient_matches_fp64_finite_differences(engine_lib):
    s = configs.microstrip(n=(32, 28, 24), n_pml=4, nt=800)
    co, pr, *_ = s.pack_inputs(gpu=True)
    out = len(pr) - 1                      # a probe of the output line voltage
    omega = 2 * np.pi * np.array([8e9, 10e9, 12e9]) * float(s.dt)
    design = FDTDDesign(s, BOX, [(0, out, 1.0)], omega, checkpoint_every=32)
    torch.manual_seed(4)
    theta = torch.randn(4, 3, 2, dtype=torch.float64, requires_grad=True)
    J = (design(1 + 9 * torch.sigmoid(theta)).abs() ** 2).sum()
    J.backward()
    g = theta.grad.numpy().copy()
    assert np.isfinite(g).all() and np.abs(g).max() > 0

    probes = km.shifted_probes(pr)
    src = np.array([p["values"][:design.nt] for p in pr], dtype=np.float64)
    J64 = _fp64_objective(design, probes, src, out, omega, 1 + 9 * torch.sigmoid(theta.detach()))
    assert abs(J64 - J.item()) <= 1e-4 * J64
    h = 1e-3
    rng = np.random.default_rng(16)
    voxels = rng.choice(g.size, size=16, replace=False)
    for flat in voxels:
        idx = np.unravel_index(flat, g.shape)
        Js = []
        for sgn in (1, -1):
            t = theta.detach().clone()
            t[idx] += sgn * h
            Js.append(_fp64_objective(design, probes, src, out, omega, 1 + 9 * torch.sigmoid(t)))
        fd = (Js[0] - Js[1]) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-3 * np.abs(g).max(), (idx, fd, g[idx])
    design.close()
