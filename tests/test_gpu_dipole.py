"""Physics bounds of the reference's dipole test, through this engine.

The reference pins its far-field path only by physics (tests/test_solver/
test_dipole.py:101-125 in the reference): a half-wave strip dipole at 10 GHz,
fed by a lumped port across its gap, meshed with d_min = 0.01 in and d_max =
0.03 in, 5-cell PML, PEC edge corrections on the strip edges, a far-field
monitor at 10 and 20 GHz. Its realized gain must stay below the theoretical
2.15 dBi and within 0.35 dB of 2.1 dBi on the theta = 90 degree circle, the
cross polarization below -40 dB, the poles below -90 dB, S11 below -10 dB and
the input resistance within 3.5 ohm of 73 ohm. The same model here runs the
time loop on the engine and the near-to-far-field transform on the GPU
(fdtd_nf2ff); the mesher is replaced by explicit graded edges with the same
feature lines and cell-size limits, built below. Their cells grow by at most
1.25 from one to the next, in the spirit of the reference mesher's blending,
which spreads the change of width to keep the growth rate low (its
utils_mesh.blend_cell_widths). With a growth of 1.5 the 20 GHz cross
polarization of this model reaches -39.5 dB; with 1.2 its cells take 66,305
distinct coefficient rows, more than the engine's 16-bit material index
addresses (the engine reports that as a size-limit error).
"""
import numpy as np
import pytest

from modelgen import geometry as geo
from modelgen import solver as S

pytestmark = pytest.mark.gpu

D_MIN, D_MAX = 0.01, 0.03


def _fill(length, d_first, d_last, growth=1.25):
    """Cell widths over `length`, growing from d_first (and, if given, back to
    d_last at the far end) by `growth`, capped at D_MAX, scaled to fit."""
    def sizes(n):
        out = []
        for k in range(n):
            a = d_first * growth ** k
            b = d_last * growth ** (n - 1 - k) if d_last else np.inf
            out.append(min(D_MAX, a, b))
        return np.array(out)
    n = 1
    while sizes(n).sum() < length:
        n += 1
    w = sizes(n)
    return w * (length / w.sum())


def _edges(lo, hi, features):
    """Graded edges over [lo, hi] through every feature coordinate, cells of
    D_MIN at the features growing to D_MAX away from them."""
    feats = sorted(set([lo, hi] + [f for f in features if lo < f < hi]))
    edges = [feats[0]]
    for a, b in zip(feats[:-1], feats[1:]):
        d_a = D_MIN if a != lo else None
        d_b = D_MIN if b != hi else None
        if d_a is None and d_b is None:
            w = _fill(b - a, D_MAX, None)
        elif d_a is None:
            w = _fill(b - a, d_b, None)[::-1]
        else:
            w = _fill(b - a, d_a, d_b)
        edges.extend(a + np.cumsum(w))
        edges[-1] = b
    return np.array(edges)


def build_dipole():
    ms_w, gap, dipole_len = 0.030, 0.015, 0.546
    sbox_len, sbox_w, sbox_h = 1.5, 1.1, 1.1
    ms_y = (-ms_w / 2, ms_w / 2)
    ms1_z = (-(dipole_len / 2), -gap / 2)
    ms2_z = (gap / 2, dipole_len / 2)
    sbox = geo.Box(bounds=(-sbox_len / 2, sbox_len / 2, -sbox_w / 2, sbox_w / 2, -sbox_h / 2, sbox_h / 2))
    s = S.FDTD_Solver(sbox)
    upper = geo.Rectangle([(0, ms_y[0], ms1_z[0]), (0, ms_y[1], ms1_z[0]), (0, ms_y[1], ms1_z[1])])
    lower = geo.Rectangle([(0, ms_y[0], ms2_z[0]), (0, ms_y[1], ms2_z[0]), (0, ms_y[1], ms2_z[1])])
    port = geo.Rectangle([(0, ms_y[0], gap / 2), (0, ms_y[1], gap / 2), (0, ms_y[1], -gap / 2)])
    s.add_conductor(upper, lower)
    s.add_lumped_port(1, port, "z-")
    s.assign_PML_boundaries("x-", "x+", "y-", "y+", "z+", "z-", n_pml=5)
    grid = (_edges(-sbox_len / 2, sbox_len / 2, [0.0]),
            _edges(-sbox_w / 2, sbox_w / 2, list(ms_y)),
            _edges(-sbox_h / 2, sbox_h / 2, [ms1_z[0], ms1_z[1], ms2_z[0], ms2_z[1]]))
    s.generate_mesh(grid=grid)
    s.add_farfield_monitor(frequency=[10e9, 20e9])
    for i, ms_z in enumerate((ms1_z, ms2_z)):
        s.edge_correction((0, ms_y[0], ms_z[0]), (0, ms_y[0], ms_z[1]), integration_line="y-")
        s.edge_correction((0, ms_y[1], ms_z[0]), (0, ms_y[1], ms_z[1]), integration_line="y+")
        s.edge_correction((0, ms_y[0], ms_z[i]), (0, ms_y[1], ms_z[i]), integration_line=("z-" if i == 0 else "z+"))
    vsrc = s.gaussian_source(width=50e-12, t0=40e-12, t_len=600e-12)
    s.assign_excitation(vsrc, 1)
    return s


def test_dipole_gain_pattern_and_match(engine_lib):
    s = build_dipole()
    s.solve(show_progress=False)
    theta, phi = np.arange(0, 190, 10), np.arange(-180, 184, 4)
    gain = s.get_farfield_gain(theta=theta, phi=phi)          # [thetapol, phipol][10, 20 GHz][theta][phi]
    gain_db = 10 * np.log10(np.maximum(gain, 1e-300))
    thetapol_90 = gain_db[0, 0, list(theta).index(90)]
    print(f"10 GHz theta=90: gain {thetapol_90.min():.3f} .. {thetapol_90.max():.3f} dBi; "
          f"cross-pol max {gain_db[1].max():.1f} dB; pole max {gain_db[0][:, [0, -1]].max():.1f} dB")
    assert np.all(thetapol_90 < 2.15)
    assert np.all(np.abs(2.1 - thetapol_90) < 0.35)
    assert np.all(gain_db[1] < -40)
    assert np.all(gain_db[0][:, [0, -1]] < -90)
    s11 = np.asarray(s.get_sparameters(np.array([10e9]), downsample=False)).reshape(-1)[0]
    z_in = 50 * (1 + s11) / (1 - s11)
    print(f"10 GHz: S11 {20 * np.log10(abs(s11)):.2f} dB, Z_in {z_in:.2f} ohm")
    assert 20 * np.log10(abs(s11)) < -10
    assert abs(73 - z_in.real) < 3.5
