"""Golden inputs of the far-field transform from the reference's own Python.

Builds a small radiating model with PML on all six faces through
rfnetwork/solver.py (the reference checkout that make_setup_golden.py
finds, with its stand-ins), adds the
far-field monitor (rfnetwork/solver.py:1777-1891), "solves" it through the
captured engine call, fills the far-field monitors with seeded random
phasors, and records what get_farfield_rE (rfnetwork/solver.py:2870-3021)
hands to core_func.nf2ff: the surface currents, cell positions and areas,
face positions and the beta / theta / phi arrays. The fixture pins
modelgen.solver's far-field monitor setup and current assembly bit for
bit; the transform itself is checked against oracle/nf2ff.py. A second
fixture, farfield_gain.npz, holds the reference's get_farfield_gain
(rfnetwork/solver.py:2804-2868) of a seeded far field, and dtft_small.npz the
reference's utils.dtft of a seeded series, plain and downsampled.

Usage:  python tests/golden/make_farfield_golden.py   (needs the reference checkout)
"""
from __future__ import annotations

import sys

import numpy as np

import make_setup_golden as mg
from modelgen import geometry as geo

FREQ = np.array([9e9, 14e9])
THETA = np.linspace(0, 180, 7)
PHI = np.linspace(0, 330, 12)


def grid_edges():
    d = 0.01
    return (np.around(np.arange(15) * d, 5), np.around(np.arange(13) * d, 5), np.around(np.arange(12) * d, 5))


def build_model(FDTD_Solver, Box, Rectangle, explicit_mesh):
    """A 0.14 x 0.12 x 0.11 in box with a short PEC dipole fed by a lumped port, PML on all faces."""
    sbox = Box(center=(0.07, 0.06, 0.055), x_length=0.14, y_length=0.12, z_length=0.11)
    s = FDTD_Solver(sbox)
    s.add_conductor(Rectangle([(0.06, 0.06, 0.03), (0.08, 0.06, 0.03), (0.08, 0.06, 0.05)]))
    s.add_conductor(Rectangle([(0.06, 0.06, 0.06), (0.08, 0.06, 0.06), (0.08, 0.06, 0.08)]))
    s.add_lumped_port(1, Rectangle([(0.06, 0.06, 0.05), (0.08, 0.06, 0.05), (0.08, 0.06, 0.06)]),
                      integration_line="z+")
    s.assign_PML_boundaries("x-", "x+", "y-", "y+", "z-", "z+", n_pml=3)
    explicit_mesh(s, grid_edges())
    s.add_farfield_monitor(FREQ, padding=1)
    src = s.gaussian_modulated_source(11e9, 150e-12, 150e-12, 60 * float(s.dt))
    s.assign_excitation(src, 1)
    return s


GAIN_POLS = ["thetapol", "phipol", "rhcp", "lhcp"]


def _install_reference_dtft(ref):
    """The reference's own utils.dtft (rfnetwork/utils.py:14-71), compiled from its
    source into the stand-in rfnetwork.utils module (the rest of utils.py needs
    pyvista and np_struct)."""
    import ast
    from scipy import signal

    src = (mg.REF / "rfnetwork/utils.py").read_text()
    fn = next(n for n in ast.parse(src).body if isinstance(n, ast.FunctionDef) and n.name == "dtft")
    ns = {"np": np, "signal": signal}
    exec(compile(ast.Module(body=[fn], type_ignores=[]), str(mg.REF / "rfnetwork/utils.py"), "exec"), ns)
    ref.utils.dtft = ns["dtft"]


def gain_field(n_freq):
    """Seeded far field rE [2, frequency, theta, phi] for the gain fixture."""
    rng = np.random.default_rng(12)
    shape = (2, n_freq, len(THETA), len(PHI))
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def monitor_values(s):
    """Seeded random phasors for the far-field monitors, by name."""
    rng = np.random.default_rng(11)
    out = {}
    for name in sorted(s.monitors):
        if name.startswith("ff_"):
            shape = s.monitors[name]["values"].shape
            out[name] = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    return out


def main():
    captured = {}
    ref = mg._install_stubs(captured)

    def nf2ff(J_xyz, M_xyz, r_grid, ds_grid, surf_pos, ff_data):
        captured["nf2ff"] = dict(J=J_xyz, M=M_xyz, r=r_grid, ds=ds_grid, pos=surf_pos, ff=ff_data)
        return 0

    ref.core.core_func.nf2ff = nf2ff
    sys.modules["pyvista"].Box = lambda bounds: geo.Box(bounds=tuple(bounds))  # the far-field box outline

    def explicit_mesh(s, edges):
        gx, gy, gz = edges
        s._create_grid = lambda d_max, d_min: setattr(s, "grid", mg._Grid(gx.astype(np.float32),
                                                                            gy.astype(np.float32),
                                                                            gz.astype(np.float32)))
        s.generate_mesh(d_max=0.01)

    s = build_model(ref.FDTD_Solver, geo.Box, geo.Rectangle, explicit_mesh)
    s.solve(n_threads=2, show_progress=False, gpu=True)
    vals = monitor_values(s)
    for name, v in vals.items():
        s.monitors[name]["values"] = v
    s.get_farfield_rE(THETA, PHI)
    c = captured["nf2ff"]
    out = {"ff_idx": np.asarray(s.farfield["idx"]), "surf_pos_m": np.asarray(s.farfield["surf_pos"])}
    for name, v in vals.items():
        out[f"mon/{name}"] = v
    for axis in range(3):
        out[f"r/{axis}/0"], out[f"r/{axis}/1"] = c["r"][axis][0], c["r"][axis][1]
        out[f"ds/{axis}"] = c["ds"][axis]
        for j in range(2):
            out[f"J/{axis}/{j}"] = c["J"][axis][j]
            out[f"M/{axis}/{j}"] = c["M"][axis][j]
            out[f"pos/{axis}/{j}"] = np.float64(c["pos"][axis][j])
    for k in ("beta", "theta", "phi"):
        out[k] = c["ff"][k]
    path = mg.HERE / "farfield_small.npz"
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({path.stat().st_size} bytes)")

    # realized gain (rfnetwork/solver.py:2804-2868) of a seeded far field: the
    # reference's own projection, port-source DTFT and normalisation
    _install_reference_dtft(ref)
    rE = gain_field(len(FREQ))
    s.get_farfield_rE = lambda theta, phi: rE
    gain = s.get_farfield_gain(THETA, PHI, polarization=GAIN_POLS)
    path = mg.HERE / "farfield_gain.npz"
    np.savez_compressed(path, rE=rE, gain=np.asarray(gain))
    print(f"wrote {path} ({path.stat().st_size} bytes)")

    # the reference's DTFT (rfnetwork/utils.py:14-71) of a seeded series, plain
    # and low-passed / decimated (downsample=True), at a time step like the models'
    rng = np.random.default_rng(13)
    x = (rng.standard_normal(4000) * np.exp(-np.linspace(0, 6, 4000))).astype(np.float32)
    f = np.linspace(1e9, 20e9, 41)
    fs = 1 / float(s.dt)
    path = mg.HERE / "dtft_small.npz"
    np.savez_compressed(path, x=x, f=f, fs=fs, X=ref.utils.dtft(x, f, fs, downsample=False),
                        X_ds=ref.utils.dtft(x, f, fs, downsample=True))
    print(f"wrote {path} ({path.stat().st_size} bytes)")


if __name__ == "__main__":
    sys.exit(main())
