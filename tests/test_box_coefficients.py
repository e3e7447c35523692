"""fdtd_set_box_coefficients patches the compiled material table in place; the
per-cell coefficients it leaves must be those a full recompile of the patched
arrays gives (host side, no GPU)."""
import numpy as np
import pytest

from modelgen import configs
from rfnetwork_b200 import _lib

NAMES = (("Ca_ex_y", "Ca_ex_z", "Cb_ex_y", "Cb_ex_z"), ("Ca_ey_z", "Ca_ey_x", "Cb_ey_z", "Cb_ey_x"),
         ("Ca_ez_x", "Ca_ez_y", "Cb_ez_x", "Cb_ez_y"))


def _expand(ids, rows):
    """Per-cell table row words [nx, ny, nz, 30] (the coefficients, flags and probe words dropped)."""
    return rows[ids.astype(np.int64)][..., :30]


def _sim(co, pr, shape, nt):
    sim = _lib.Simulation(*shape)
    sim.set_coefficients(co)
    for p in pr:
        sim.add_probe(p["field"], p["idx"], p["is_source"], p["values"][:nt] if p["is_source"] else None)
    return sim


def _patched(co, box, coefs):
    out = {k: v.copy() for k, v in co.items()}
    sl = (slice(box[0], box[1]), slice(box[2], box[3]), slice(box[4], box[5]))
    for c, (ca1, ca2, cb1, cb2) in enumerate(NAMES):
        for name, k in ((ca1, 0), (ca2, 0), (cb1, 1), (cb2, 2)):
            out[name][sl] = coefs[c, k]
    return out


def _coefs(co, box, seed):
    rng = np.random.default_rng(seed)
    sl = (slice(box[0], box[1]), slice(box[2], box[3]), slice(box[4], box[5]))
    base = np.stack([np.stack([co[n[0]][sl], co[n[2]][sl], co[n[3]][sl]]) for n in NAMES])
    return (base * (1 + 0.2 * rng.random(base.shape))).astype(np.float32)


def test_box_patch_matches_full_recompile(engine_lib):
    s = configs.microstrip(n=(20, 18, 14), n_pml=3, nt=50)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)
    sim = _sim(co, pr, (Nx, Ny, Nz), Nt)
    sim.compile()
    cur = co
    for box, seed in (((7, 11, 6, 9, 4, 7), 1), ((7, 11, 6, 9, 4, 7), 2), ((8, 12, 7, 11, 5, 8), 3)):
        coefs = _coefs(cur, box, seed)
        sim.set_box_coefficients(box, coefs)
        cur = _patched(cur, box, coefs)
        ref = _sim(cur, pr, (Nx, Ny, Nz), Nt)
        a, b = _expand(*sim.material_table()), _expand(*ref.material_table())
        ref.close()
        assert np.array_equal(a, b)
    # a full recompile of the simulation's own arrays agrees as well
    sim.set_coefficient("Ca_ex_y", cur["Ca_ex_y"])
    assert np.array_equal(_expand(*sim.material_table()), b)
    sim.close()


def test_box_patch_rejects_split_cells(engine_lib):
    s = configs.microstrip(n=(20, 18, 14), n_pml=3, nt=50)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)
    sim = _sim(co, pr, (Nx, Ny, Nz), Nt)
    sim.compile()
    box = (0, 4, 6, 9, 4, 7)   # reaches into the x PML
    with pytest.raises(ValueError, match="split"):
        sim.set_box_coefficients(box, _coefs(co, box, 0))
    sim.close()
