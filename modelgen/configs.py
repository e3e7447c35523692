"""Synthetic FDTD workloads used by the benchmark and the parity tests.

Every model is built through the ``FDTD_Solver`` setup API, so the engine sees
the same coefficient arrays the reference's ``solve()`` would pass. Cells are
uniform cubes of 2**-7 inch (0.198 mm): the float32 cell width closest to
0.2 mm whose grid coordinates and widths are exact in float32, so the grid is
truly uniform (a 0.2 mm grid in inches is not representable and its float32
widths would differ in the last bits from cell to cell).
"""
from __future__ import annotations

import numpy as np

from . import geometry as geo
from .solver import FDTD_Solver

D = 2.0 ** -7  # cell width, inches


def _grid(n):
    return [np.arange(k + 1) * D for k in n]


def _coarsened(k, spans):
    """Uniform edges 0..k (cells of D) with every other edge dropped inside
    the given [a, b) cell spans: cells of 2D there, D elsewhere."""
    drop = set()
    for a, b in spans:
        drop.update(range(a + 1, b, 2))
    return np.array([i * D for i in range(k + 1) if i not in drop])


def microstrip(n=(64, 64, 48), n_pml=10, nt=2000, courant=0.99, graded=False):
    """Plain microstrip model (64x64x48, 10-cell PML on all faces, 2000 steps).

    eps_r = 3.0 substrate, 4 cells thick, on a PEC ground sheet; PEC strip 6
    cells wide and 1 cell thick along x over 40 cells; 50-ohm lumped ports
    at both strip ends (port 1 driven with a Gaussian-modulated sinusoid,
    10 GHz centre, 16 GHz bandwidth); line voltage probes at both ends.
    Smaller ``n`` keeps the layout proportions for quick tests. ``graded``
    coarsens the mesh to 2-cell widths in the air above the strip and towards
    the y sides (every feature plane stays a cell edge), for a non-uniform grid.
    """
    nx, ny, nz = n
    s = FDTD_Solver(geo.Box(bounds=(0, nx * D, 0, ny * D, 0, nz * D)), courant=courant)
    zg = n_pml + max(2, nz // 12)          # ground plane height (cells)
    zs = zg + 4                            # strip bottom
    yc = ny // 2
    w = 6 if ny >= 24 else 2
    y0, y1 = yc - w // 2, yc - w // 2 + w
    xlen = min(40, nx - 2 * n_pml - 4) if nx >= 2 * n_pml + 8 else nx - 4
    x0 = (nx - xlen) // 2
    x1 = x0 + xlen
    s.add_dielectric(geo.Box(bounds=(0, nx * D, 0, ny * D, zg * D, zs * D)), er=3.0)
    s.add_conductor(geo.Rectangle([(0, 0, zg * D), (nx * D, 0, zg * D), (nx * D, ny * D, zg * D)]))
    s.add_conductor(geo.Box(bounds=(x0 * D, x1 * D, y0 * D, y1 * D, zs * D, (zs + 1) * D)))
    for k, xp in ((1, x0), (2, x1)):
        face = geo.Rectangle([(xp * D, y0 * D, zs * D), (xp * D, y1 * D, zs * D), (xp * D, y1 * D, zg * D)])
        s.add_lumped_port(k, face, integration_line="z+")
    if n_pml:
        s.assign_PML_boundaries("x-", "x+", "y-", "y+", "z-", "z+", n_pml=n_pml)
    if graded:
        grid = [np.arange(nx + 1) * D,
                _coarsened(ny, [(n_pml + 1, y0 - 1), (y1 + 1, ny - n_pml - 1)]),
                _coarsened(nz, [(zs + 3, nz - n_pml - 1)])]
    else:
        grid = _grid(n)
    s.generate_mesh(grid=grid)
    for name, xp in (("v1", x0 + 1), ("v2", x1 - 1)):
        s.add_voltage_probe(name, geo.Line(((xp + 0.5) * D, yc * D, zs * D), ((xp + 0.5) * D, yc * D, zg * D)))
    f0, bw = 10e9, 16e9
    tau = 1 / (np.pi * bw / 2)             # spectral envelope 1/e at f0 +- bw/2
    width = 4 * tau
    vsrc = s.gaussian_modulated_source(f0, width, width, (nt + 0.5) * float(s.dt))
    s.assign_excitation(vsrc, 1)
    return s


def microstrip_frequencies(n=101):
    return np.linspace(1e9, 20e9, n)


def boxes(n=(256, 256, 128), n_pml=8, n_boxes=64, nt=5000, seed=2, n_ports=4, n_probes=16, courant=0.99):
    """Bandwidth model: 64 seeded dielectric boxes in free space.

    Each box edge is 8-64 cells (clipped to the interior), eps_r ~ U[1, 10],
    sigma ~ U[0, 0.05] S/m; 4 lumped 50-ohm ports (4x4-cell faces normal to x,
    integration z+) driven by a Gaussian pulse; 16 Ez point probes; 8-cell PML
    on all faces.
    """
    rng = np.random.default_rng(seed)
    nx, ny, nz = n
    s = FDTD_Solver(geo.Box(bounds=(0, nx * D, 0, ny * D, 0, nz * D)), courant=courant)
    lo = np.array([n_pml + 1] * 3)
    hi = np.array(n) - n_pml - 1
    span = hi - lo
    f_sig = 1e9
    for b in range(n_boxes):
        size = np.minimum(rng.integers(8, 65, size=3), span)
        start = lo + np.array([rng.integers(0, span[a] - size[a] + 1) for a in range(3)])
        er = rng.uniform(1.0, 10.0)
        sigma = rng.uniform(0.0, 0.05)
        loss_tan = sigma / (8.854187817e-12 * er * 2 * np.pi * f_sig)
        bnd = tuple(v for a in range(3) for v in (start[a] * D, (start[a] + size[a]) * D))
        s.add_dielectric(geo.Box(bounds=bnd), er=er, loss_tan=loss_tan, f0=f_sig)
    for k in range(n_ports):
        px = int(rng.integers(lo[0] + 2, hi[0] - 2))
        py = int(rng.integers(lo[1] + 2, hi[1] - 6))
        pz = int(rng.integers(lo[2] + 2, hi[2] - 6))
        face = geo.Rectangle([(px * D, py * D, (pz + 4) * D), (px * D, (py + 4) * D, (pz + 4) * D),
                              (px * D, (py + 4) * D, pz * D)])
        s.add_lumped_port(k + 1, face, integration_line="z+")
    if n_pml:
        s.assign_PML_boundaries("x-", "x+", "y-", "y+", "z-", "z+", n_pml=n_pml)
    s.generate_mesh(grid=_grid(n))
    for k in range(n_probes):
        idx = [int(rng.integers(lo[a] + 1, hi[a] - 1)) for a in range(3)]
        s.add_point_probe(f"pz{k}", "ez", idx)
    width = 120e-12
    vsrc = s.gaussian_source(width, width, (nt + 0.5) * float(s.dt))
    s.assign_excitation(vsrc, list(range(1, n_ports + 1)))
    return s


def boxes_frequencies(n=51):
    return np.linspace(1e9, 25e9, n)


def batch_member(seed: int, i: int, n_pml=8, nt=3000, size_range=(32, 160), n_boxes=8, n_probes=4, courant=0.99):
    """One simulation of the batched workload: grid axes ~ U{32..160}, 8 boxes
    eps_r ~ U[1, 10], one Gaussian point source on Ez at a random interior cell,
    4 Ez point probes."""
    rng = np.random.default_rng([seed, i])
    n = tuple(int(v) for v in rng.integers(size_range[0], size_range[1] + 1, size=3))
    s = FDTD_Solver(geo.Box(bounds=(0, n[0] * D, 0, n[1] * D, 0, n[2] * D)), courant=courant)
    lo = np.array([n_pml + 1] * 3)
    hi = np.array(n) - n_pml - 1
    span = hi - lo
    for b in range(n_boxes):
        size = np.minimum(rng.integers(4, 33, size=3), span)
        start = lo + np.array([rng.integers(0, span[a] - size[a] + 1) for a in range(3)])
        bnd = tuple(v for a in range(3) for v in (start[a] * D, (start[a] + size[a]) * D))
        s.add_dielectric(geo.Box(bounds=bnd), er=rng.uniform(1.0, 10.0))
    s.assign_PML_boundaries("x-", "x+", "y-", "y+", "z-", "z+", n_pml=n_pml)
    s.generate_mesh(grid=_grid(n))
    src_idx = [int(rng.integers(lo[a] + 1, hi[a] - 1)) for a in range(3)]
    width = 120e-12
    vsrc = s.gaussian_source(width, width, (nt + 0.5) * float(s.dt)).astype(np.float32)
    s.add_soft_source("src", "ez", src_idx, vsrc[:nt])
    for k in range(n_probes):
        idx = [int(rng.integers(lo[a] + 1, hi[a] - 1)) for a in range(3)]
        s.add_point_probe(f"pz{k}", "ez", idx)
    return s


def pml_cells(n, n_pml, sides=6):
    """Cells inside the PML slabs of a grid with PML on all six faces."""
    nx, ny, nz = n
    inner = max(nx - 2 * n_pml, 0) * max(ny - 2 * n_pml, 0) * max(nz - 2 * n_pml, 0)
    return nx * ny * nz - inner


def algorithmic_bytes(n, n_pml):
    """Algorithmic HBM bytes of one time step: 49 B per interior cell-update
    (6 fields read + written, 1 B material index) and 97 B per PML cell-update
    (12 split components read + written, 1 B index)."""
    total = n[0] * n[1] * n[2]
    p = pml_cells(n, n_pml)
    return 49 * (total - p) + 97 * p
