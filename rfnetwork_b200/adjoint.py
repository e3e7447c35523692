"""Gradients of DFT objectives with respect to a permittivity / conductivity design.

``FDTDDesign`` wraps one model and a box of design cells. The model is what
the reference's ``FDTD_Solver.solve()`` hands its engine (the packed
coefficient dict, the probe list, the grid shape and the number of steps,
rfnetwork/solver.py:1441-1575) plus the cell material it was built from
(``dt``, ``eps``, ``sigma``, ``d_cells``): a ``PackedModel``, or any object
with a ``pack_inputs(gpu=True)`` method and those attributes. Called with the
relative permittivity (and optionally the conductivity) of the design cells as
torch tensors, it returns the complex device DFT of the chosen probe series as
a torch tensor that autograd can differentiate:

    design = FDTDDesign(model, (x0, x1, y0, y1, z0, z1), terms, omega)
    X = design(1 + 9 * torch.sigmoid(theta))          # complex [series, frequency]
    J = (X.abs() ** 2).sum()
    J.backward()                                        # theta.grad

Forward: the design cells' permittivity is averaged onto the E-field sites as
the solver does (edge averages weighted by half cell widths, the reference's
average_cells, rfnetwork/solver.py:892-912), turned into the update
coefficients Ca = (2 eps - sigma dt) / (2 eps + sigma dt) and
Cb = 2 dt / (2 eps + sigma dt) (rfnetwork/solver.py:954-961), scaled by the
packing's inverse cell widths, and the engine runs the time loop keeping what
the adjoint needs: by default the forward history of the gradient box at every
step (fdtd_run_recorded; 36 bytes per box cell per step), or, when that would
exceed ``history_budget`` bytes or ``checkpoint_every`` is given, a field
snapshot every ``checkpoint_every`` (default ~sqrt(nt)) steps
(fdtd_run_checkpointed), from which the adjoint recomputes each segment.
Backward: the engine's discrete adjoint (fdtd_adjoint) returns dJ/d(Ca, Cb) of
the affected E sites; torch chains them to the design tensors.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch

from ._lib import Batch, Simulation
from .solver_constants import COEFF_NAMES
from .units import conv

E0 = 8.854187817e-12

# per E component: the Ca name whose twin must stay equal, and the two Cb names
_CA = (("Ca_ex_y", "Ca_ex_z"), ("Ca_ey_z", "Ca_ey_x"), ("Ca_ez_x", "Ca_ez_y"))
_CB = (("Cb_ex_y", "Cb_ex_z"), ("Cb_ey_z", "Cb_ey_x"), ("Cb_ez_x", "Cb_ez_y"))
# cells whose permittivity an E site of each component averages (offsets in
# the packed index space of the coefficient arrays; see pack_inputs)
_AVG = (((0, 0), (0, 1), (0, 1)), ((0, 1), (0, 0), (0, 1)), ((0, 1), (0, 1), (0, 0)))


class _Run(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coefs, design):
        ctx.design = design
        return torch.from_numpy(design._run(coefs.detach().cpu().numpy()))

    @staticmethod
    def backward(ctx, gX):
        g = ctx.design.sim.adjoint(gX.detach().cpu().numpy(), ctx.design.box)
        return torch.from_numpy(g), None


@dataclass
class PackedModel:
    """The engine inputs of one model and the material they were built from.

    coefficients: the 30 float32 (Nx, Ny, Nz) arrays keyed as the reference's
    packing names them (rfnetwork/solver.py:1473-1518); probes: its probe
    dicts (``values``, ``field``, ``idx``, ``is_source``); shape (Nx, Ny, Nz);
    nt time steps; dt seconds; eps, sigma: per-cell permittivity (F/m) and
    conductivity (S/m), shape (Nx, Ny, Nz); d_cells: cell widths per axis in
    inches, as the reference's ``FDTD_Solver.d_cells``.
    """
    coefficients: dict
    probes: list
    shape: tuple
    nt: int
    dt: float
    eps: np.ndarray
    sigma: np.ndarray
    d_cells: tuple

    @classmethod
    def of(cls, model) -> "PackedModel":
        """A PackedModel as is, or one read off an object with ``pack_inputs``."""
        if isinstance(model, cls):
            return model
        co, pr, mo, mem, Nx, Ny, Nz, Nt = model.pack_inputs(gpu=True)
        return cls(co, pr, (Nx, Ny, Nz), Nt, float(model.dt), model.eps, model.sigma, tuple(model.d_cells))


class FDTDDesign:
    """A model whose design cells' material enters the time loop differentiably."""

    def __init__(self, model, design_box, terms, omega, checkpoint_every: int | None = None,
                 history_budget: float = 8 * 2**30):
        m = PackedModel.of(model)
        co, pr, (Nx, Ny, Nz), Nt = m.coefficients, m.probes, m.shape, m.nt
        self.shape = (Nx, Ny, Nz)
        self.nt = Nt
        self.base = {k: np.ascontiguousarray(v, dtype=np.float32) for k, v in co.items()}
        x0, x1, y0, y1, z0, z1 = [int(v) for v in design_box]
        self.design_box = (x0, x1, y0, y1, z0, z1)
        # E sites whose average touches a design cell sit at most one cell below it
        self.box = (max(x0 - 1, 0), min(x1, Nx), max(y0 - 1, 0), min(y1, Ny), max(z0 - 1, 0), min(z1, Nz))
        bx0, bx1, by0, by1, bz0, bz1 = self.box
        history_bytes = 36 * (bx1 - bx0) * (by1 - by0) * (bz1 - bz0) * Nt
        self.recorded = checkpoint_every is None and history_bytes <= history_budget
        self.checkpoint_every = None if self.recorded else int(checkpoint_every or max(1, round(math.sqrt(Nt))))
        self.probes = pr  # the probe dicts of the packing (source amplitudes, fields, indices)
        self.sim = Simulation(Nx, Ny, Nz)
        self.sim.set_coefficients(self.base)
        for p in pr:
            src = bool(p["is_source"])
            self.sim.add_probe(int(p["field"]), p["idx"], src, p["values"][:Nt] if src else None)
        self.sim.set_dft(terms, omega)
        self.dt = float(m.dt)
        # cell material and half widths around the box (float64), one cell of margin above
        sl = (slice(bx0, min(bx1 + 1, Nx)), slice(by0, min(by1 + 1, Ny)), slice(bz0, min(bz1 + 1, Nz)))
        self._sl = sl
        self._eps = torch.from_numpy(np.asarray(m.eps, dtype=np.float64)[sl].copy())
        self._sig = torch.from_numpy(np.asarray(m.sigma, dtype=np.float64)[sl].copy())
        self._d = [torch.from_numpy(np.asarray(conv.m_in(d), dtype=np.float64)[s].copy())
                   for d, s in zip(m.d_cells, sl)]
        # design cells inside the margin array
        self._dsl = (slice(x0 - bx0, x1 - bx0), slice(y0 - by0, y1 - by0), slice(z0 - bz0, z1 - bz0))
        # the packing's scale of each Cb (inverse widths and sign), read off the base model
        eps_b, sig_b = self._site_material(self._eps, self._sig)
        self._scale, self._touch, self._base_t = [], [], []
        box_sl = (slice(bx0, bx1), slice(by0, by1), slice(bz0, bz1))
        dmask = torch.zeros_like(self._eps, dtype=torch.bool)
        dmask[self._dsl] = True
        for c in range(3):
            cb = (2 * self.dt / (2 * eps_b[c] + sig_b[c] * self.dt)).numpy()
            s1 = self.base[_CB[c][0]][box_sl].astype(np.float64) / cb
            s2 = self.base[_CB[c][1]][box_sl].astype(np.float64) / cb
            self._scale.append((torch.from_numpy(s1), torch.from_numpy(s2)))
            self._touch.append(self._average(dmask.double(), c) > 0)
            self._base_t.append(torch.from_numpy(np.stack(
                [self.base[_CA[c][0]][box_sl], self.base[_CB[c][0]][box_sl], self.base[_CB[c][1]][box_sl]]
            ).astype(np.float64)))

    # ------------------------------------------------------------- material
    def _average(self, v, c):
        """Half-width weighted average of cell values v onto the box's E sites of component c."""
        bx0, bx1, by0, by1, bz0, bz1 = self.box
        out = v
        for ax in range(3):
            lo, hi = _AVG[c][ax]
            n = (bx1 - bx0, by1 - by0, bz1 - bz0)[ax]
            if hi == 0:
                out = out.narrow(ax, 0, n)
                continue
            d = self._d[ax]
            a, b = out.narrow(ax, 0, n), out.narrow(ax, 1, n)
            shp = [1, 1, 1]
            shp[ax] = n
            da, db = d[:n].reshape(shp), d[1:n + 1].reshape(shp)
            out = (a * (da / 2) + b * (db / 2)) / (da / 2 + db / 2)
        return out

    def _site_material(self, eps, sig):
        return [self._average(eps, c) for c in range(3)], [self._average(sig, c) for c in range(3)]

    def coefficients(self, eps_r, sigma=None):
        """(Ca, Cb1, Cb2) of each E component on the gradient box, [3, 3, *box], from the design cells."""
        eps = self._eps.clone()
        eps[self._dsl] = E0 * eps_r.to(torch.float64)
        sig = self._sig.clone()
        if sigma is not None:
            sig[self._dsl] = sigma.to(torch.float64)
        eps_s, sig_s = self._site_material(eps, sig)
        out = []
        for c in range(3):
            den = 2 * eps_s[c] + sig_s[c] * self.dt
            ca = (2 * eps_s[c] - sig_s[c] * self.dt) / den
            cb = 2 * self.dt / den
            vals = torch.stack([ca, cb * self._scale[c][0], cb * self._scale[c][1]])
            # sites no design cell touches keep their coefficients bit for bit
            out.append(torch.where(self._touch[c], vals, self._base_t[c]))
        return torch.stack(out)

    # -------------------------------------------------------------- running
    def _set(self, coefs: np.ndarray):
        # both Ca twins take the same value on the box, so its sites stay unsplit;
        # once compiled, the engine patches its material table in place
        self.sim.set_box_coefficients(self.box, coefs)

    def _run(self, coefs: np.ndarray) -> np.ndarray:
        self._set(coefs)
        if self.recorded:
            self.sim.run_recorded(self.nt, self.box)
        else:
            self.sim.run_checkpointed(self.nt, self.checkpoint_every)
        return self.sim.dft()

    def forward_only(self, eps_r, sigma=None) -> np.ndarray:
        """The same forward solve without snapshots (no gradient), for comparison."""
        with torch.no_grad():
            self._set(self.coefficients(eps_r, sigma).numpy())
        self.sim.run(self.nt)
        return self.sim.dft()

    def __call__(self, eps_r, sigma=None):
        return _Run.apply(self.coefficients(eps_r, sigma), self)

    def close(self):
        self.sim.close()


class _RunBatch(torch.autograd.Function):
    @staticmethod
    def forward(ctx, coefs, design):
        ctx.design = design
        return torch.from_numpy(design._run(coefs.detach().cpu().numpy()))

    @staticmethod
    def backward(ctx, gX):
        g = ctx.design.batch.adjoint(list(gX.detach().cpu().numpy()))
        return torch.from_numpy(np.stack(g)), None


class FDTDDesignBatch:
    """Several designs (variants of models, one design box each) whose forward
    solves run as one batch and whose adjoints run as one batched sweep.

        designs = FDTDDesignBatch([model] * 32, box, terms, omega)
        X = designs([1 + 9 * torch.sigmoid(t) for t in thetas])   # complex [member, series, freq]

    As for one design, the members keep the box history of their forward run
    (fdtd_batch_run_recorded) while all histories together fit
    ``history_budget`` bytes and ``checkpoint_every`` is not given; otherwise
    each member's state is snapshot every ``checkpoint_every`` (default
    ~sqrt(nt)) steps (fdtd_batch_run_checkpointed) and the batched adjoint
    replays the segments of all members together. The gradient boxes must have
    one shape so the coefficients stack."""

    def __init__(self, models, design_box, terms, omega, checkpoint_every: int | None = None,
                 history_budget: float = 8 * 2**30):
        self.members = [FDTDDesign(m, design_box, terms, omega, checkpoint_every=None, history_budget=float("inf"))
                        for m in models]
        shapes = {tuple(b - a for a, b in zip(m.box[0::2], m.box[1::2])) for m in self.members}
        if len(shapes) != 1 or len({m.nt for m in self.members}) != 1:
            raise ValueError("batch members need one gradient-box shape and one number of time steps")
        self.nt = self.members[0].nt
        bx0, bx1, by0, by1, bz0, bz1 = self.members[0].box
        history_bytes = 36 * (bx1 - bx0) * (by1 - by0) * (bz1 - bz0) * self.nt * len(self.members)
        self.recorded = checkpoint_every is None and history_bytes <= history_budget
        self.checkpoint_every = None if self.recorded else int(checkpoint_every or max(1, round(math.sqrt(self.nt))))
        self.batch = Batch([m.sim for m in self.members])

    def _run(self, coefs: np.ndarray) -> np.ndarray:
        for m, c in zip(self.members, coefs):
            m._set(c)
        boxes = [m.box for m in self.members]
        if self.recorded:
            self.batch.run_recorded(self.nt, boxes)
        else:
            self.batch.run_checkpointed(self.nt, self.checkpoint_every, boxes)
        return np.stack([m.sim.dft() for m in self.members])

    def __call__(self, eps_r, sigma=None):
        sig = sigma if sigma is not None else [None] * len(self.members)
        coefs = torch.stack([m.coefficients(e, g) for m, e, g in zip(self.members, eps_r, sig)])
        return _RunBatch.apply(coefs, self)

    def close(self):
        self.batch.close()
        for m in self.members:
            m.close()


__all__ = ["PackedModel", "FDTDDesign", "FDTDDesignBatch", "COEFF_NAMES"]
