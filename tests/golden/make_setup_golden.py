"""Generate golden setup fixtures from the reference's own Python setup code.

Runs rfnetwork/solver.py from the reference checkout (the location the
oracle's build recipe uses: oracle/ref_cuda.py ``REF_ROOT``, which
$RFN_REFERENCE_ROOT overrides) and records exactly what
``FDTD_Solver.solve()`` hands to the engine (the coefficient dict, probe list
and monitor list of rfnetwork/solver.py:1473-1641), for the CPU and the GPU
packing. The reference's third-party imports that are absent here
(pyvista, np_struct, skimage, matplotlib, the compiled core) are replaced by
minimal stand-ins:
  * pyvista objects carry only ``points`` / ``n_cells`` / ``faces`` / ``bounds``;
  * ``_create_grid`` (the mesher, out of scope) is replaced by explicit grid
    edges: uniform (setup_small.npz, and setup_edge.npz, which adds the PEC
    edge corrections of the trace) or graded (setup_graded.npz);
  * the conductor inclusion tests use axis-aligned box / rectangle
    containment (``utils_mesh.is_point_in_surface`` and pyvista's implicit
    distance are geometry code, not coefficient math).
Everything else -- grid arrays, material averaging, coefficients, PML,
conductors, lumped ports, probes, monitors, sources and packing -- is the
reference code itself. The fixture pins ``modelgen.solver`` bit-exactly.

Usage:  python tests/golden/make_setup_golden.py [setup_small.npz] [setup_graded.npz] [setup_edge.npz]
        (needs the reference checkout; writes the named fixtures, default both)
"""
from __future__ import annotations

import importlib.util
import os
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))
from oracle.ref_cuda import REF_ROOT as REF  # noqa: E402  (the one place that names the checkout)

from modelgen import geometry as geo  # noqa: E402  (stand-in geometry shared with the mirror)


# --------------------------------------------------------------- stand-ins
class _PolyData:
    def __init__(self, points=None):
        self.points = np.asarray(points, dtype=np.float32) if points is not None else np.zeros((0, 3), np.float32)

    def compute_implicit_distance(self, obj):
        return {"implicit_distance": obj.implicit_distance(self.points.astype(float))}


class _Grid:
    def __init__(self, x, y, z):
        self.x, self.y, self.z = np.asarray(x), np.asarray(y), np.asarray(z)


def _install_stubs(captured):
    pv = types.ModuleType("pyvista")
    pv.PolyData = _PolyData
    pv.RectilinearGrid = _Grid
    pv.Rectangle = lambda pts: geo.Rectangle(pts)
    pv.Cube = lambda center=(0, 0, 0), x_length=1, y_length=1, z_length=1: geo.Box(center, x_length, y_length,
                                                                                     z_length)
    pv.Line = lambda a, b: geo.Line(a, b)
    for unused in ("Plotter", "CameraPosition", "ImageData", "Box"):   # only named in annotations
        setattr(pv, unused, object)
    sys.modules["pyvista"] = pv

    nps = types.ModuleType("np_struct")
    nps.ldarray = lambda data, coords=None, **kw: np.asarray(data)
    sys.modules["np_struct"] = nps

    for name in ("skimage", "matplotlib", "matplotlib.axes", "matplotlib.colors", "matplotlib.pyplot"):
        mod = types.ModuleType(name)
        sys.modules[name] = mod
    sys.modules["matplotlib.axes"].Axes = object

    pkg = types.ModuleType("rfnetwork")
    pkg.__path__ = [str(REF / "rfnetwork")]
    sys.modules["rfnetwork"] = pkg

    units = _load("rfnetwork.core.units", REF / "rfnetwork/core/units.py")
    pkg.const, pkg.conv = units.const, units.conv

    utils_mesh = types.ModuleType("rfnetwork.utils_mesh")
    utils_mesh.is_object_surface = geo.is_object_surface
    utils_mesh.is_point_in_surface = lambda points, obj, tolerance=0.1, d_min=None: geo.points_in_rectangle(
        points, obj, 1e-5)
    pkg.utils_mesh = utils_mesh

    utils = types.ModuleType("rfnetwork.utils")
    pkg.utils = utils

    def capture(kind):
        def run(coefficients, probes, monitors, mem, Nx, Ny, Nz, Nt, n_threads, update_interval):
            captured[kind] = dict(coefficients=coefficients, probes=probes, monitors=monitors, mem_size=mem.size,
                                  N=(Nx, Ny, Nz, Nt))
            return 0
        return run

    core = types.SimpleNamespace(
        cuda_func=types.SimpleNamespace(solver_run_cu=capture("gpu")),
        core_func=types.SimpleNamespace(solver_run=capture("cpu")),
    )
    pkg.core = core
    return _load("rfnetwork.solver", REF / "rfnetwork/solver.py")


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


# ------------------------------------------------------------- the model
def build_model(FDTD_Solver, Box, Rectangle, Line, grid_edges, explicit_mesh):
    """Small microstrip-like model exercising every setup path of the FDTD slice."""
    d = 0.01
    sbox = Box(center=(0.08, 0.06, 0.05), x_length=0.16, y_length=0.12, z_length=0.10)
    s = FDTD_Solver(sbox)
    sub = Box(center=(0.08, 0.06, 0.01), x_length=0.16, y_length=0.12, z_length=0.02)
    s.add_dielectric(sub, er=3.66, loss_tan=0.01, f0=10e9)
    blk = Box(center=(0.10, 0.05, 0.04), x_length=0.04, y_length=0.04, z_length=0.02)
    s.add_dielectric(blk, er=6.0)
    trace = Rectangle([(0.03, 0.05, 0.02), (0.03, 0.07, 0.02), (0.13, 0.07, 0.02)])
    s.add_conductor(trace)
    pec_box = Box(center=(0.08, 0.06, 0.075), x_length=0.02, y_length=0.02, z_length=0.01)
    s.add_conductor(pec_box, sigma=5.8e7)
    port1 = Rectangle([(0.03, 0.05, 0.02), (0.03, 0.07, 0.02), (0.03, 0.07, 0.0)])
    s.add_lumped_port(1, port1, integration_line="z+")
    port2 = Rectangle([(0.13, 0.05, 0.02), (0.13, 0.07, 0.02), (0.13, 0.07, 0.0)])
    s.add_lumped_port(2, port2, integration_line="z-")
    res = Rectangle([(0.06, 0.09, 0.02), (0.08, 0.09, 0.02), (0.08, 0.09, 0.0)])
    s.add_resistor(res, 100.0, "z+")
    s.assign_PML_boundaries("x+", "y-", "z+", n_pml=3)
    explicit_mesh(s, grid_edges)
    s.add_voltage_probe("v1", Line((0.08, 0.06, 0.02), (0.08, 0.06, 0.0)))
    s.add_current_probe("c1", Rectangle([(0.079, 0.049, 0.021), (0.079, 0.071, 0.021), (0.079, 0.071, 0.019)]))
    s.add_field_monitor("mz", "ez", "z", index=1, n_step=3)
    s.add_field_monitor("mx", "hy", "x", index=5, n_step=1, frequency=np.array([5e9, 9e9]))
    s.add_field_monitor("my", "ex", "y", index=4, n_step=2)
    src = s.gaussian_modulated_source(10e9, 150e-12, 150e-12, 120 * float(s.dt))
    s.assign_excitation(src, 1)
    return s


def grid_edges():
    d = 0.01
    return (np.around(np.arange(17) * d, 5), np.around(np.arange(13) * d, 5), np.around(np.arange(11) * d, 5))


def grid_edges_graded():
    """Non-uniform edges for the same model: 0.005 / 0.01 / 0.015 / 0.02 cells
    that keep every feature plane of build_model on a cell edge, with uniform
    cells in the PML layers (x+, y-, z+)."""
    gx = [0, 0.02, 0.03, 0.035, 0.04, 0.05, 0.06, 0.07, 0.075, 0.08, 0.085, 0.09, 0.10, 0.11, 0.12, 0.13,
          0.14, 0.15, 0.16]
    gy = [0, 0.01, 0.02, 0.03, 0.04, 0.05, 0.055, 0.06, 0.065, 0.07, 0.08, 0.09, 0.105, 0.12]
    gz = [0, 0.01, 0.015, 0.02, 0.03, 0.05, 0.06, 0.07, 0.08, 0.09, 0.10]
    return tuple(np.around(np.array(g), 5) for g in (gx, gy, gz))


# PEC edge corrections on the trace (rfnetwork/solver.py:2534-2700): both long
# edges along x, pointing away from the strip in the substrate plane, and the
# far end of the strip along y
TRACE_EDGES = [((0.03, 0.05, 0.02), (0.13, 0.05, 0.02), "y-"),
               ((0.13, 0.07, 0.02), (0.03, 0.07, 0.02), "y+"),
               ((0.13, 0.05, 0.02), (0.13, 0.07, 0.02), "x+")]


def with_edge_corrections(s):
    for p1, p2, line in TRACE_EDGES:
        s.edge_correction(p1, p2, line)
    return s


FIXTURES = {"setup_small.npz": grid_edges, "setup_graded.npz": grid_edges_graded, "setup_edge.npz": grid_edges}
# applied to the built and meshed model before it is solved
POST_BUILD = {"setup_edge.npz": with_edge_corrections}


def main(names):
    for name in names:
        generate(name, FIXTURES[name]())


def generate(name, edges):
    captured = {}
    ref = _install_stubs(captured)

    def explicit_mesh(s, edges):
        gx, gy, gz = edges

        def fake_create_grid(d_max, d_min):
            s.grid = _Grid(gx.astype(np.float32), gy.astype(np.float32), gz.astype(np.float32))

        s._create_grid = fake_create_grid
        s.generate_mesh(d_max=0.01)

    s = build_model(ref.FDTD_Solver, geo.Box, geo.Rectangle, geo.Line, edges, explicit_mesh)
    POST_BUILD.get(name, lambda m: m)(s)
    s.solve(n_threads=2, show_progress=False, gpu=False)
    s.solve(n_threads=2, show_progress=False, gpu=True)

    out = {"dt": np.float32(s.dt), "N": np.array(captured["gpu"]["N"])}
    for kind in ("cpu", "gpu"):
        c = captured[kind]
        for k, v in c["coefficients"].items():
            out[f"{kind}/coef/{k}"] = v
        for i, p in enumerate(c["probes"]):
            out[f"{kind}/probe/{i}/values"] = p["values"]
            out[f"{kind}/probe/{i}/meta"] = np.array([p["field"], *p["idx"], p["is_source"]])
        for i, m in enumerate(c["monitors"]):
            out[f"{kind}/monitor/{i}/meta"] = np.array([m["axis"], m["position"], m["field"], m["n_step"]])
            out[f"{kind}/monitor/{i}/shape"] = np.array(m["values"].shape)
            if "dtft_phase" in m:
                out[f"{kind}/monitor/{i}/dtft_phase"] = m["dtft_phase"]
        out[f"{kind}/mem_size"] = np.array(c["mem_size"])
    # port records and probe widths (used by the S-parameter post-processing)
    for i, p in enumerate(s.ports):
        out[f"port/{i}/Vs_a"] = np.asarray(p["Vs_a"])
        out[f"port/{i}/meta"] = np.array([p["axis"], p["r0"], p["direction"]])
    out["probe_d"] = np.array([p["d"] for p in s.probes.values()], dtype=np.float64)
    out["probe_names"] = np.array(list(s.probes.keys()))
    path = HERE / name
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({path.stat().st_size} bytes), {len(captured['gpu']['probes'])} probes")


if __name__ == "__main__":
    main(sys.argv[1:] or list(FIXTURES))
