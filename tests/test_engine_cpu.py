"""Engine library checks that need no GPU: it loads, exports every declared
entry point, validates arguments, and its host-side material-table compiler
reproduces the oracle's arithmetic (replayed through tests/kernel_model.py)."""
import re

import numpy as np
import pytest

import kernel_model as km
import make_setup_golden as mg
from helpers import rel_l2, run_oracle
from modelgen import configs
from rfnetwork_b200 import _lib
from modelgen import geometry as geo
from modelgen import solver as S
from rfnetwork_b200.solver_constants import COEFF_NAMES

HEADER = mg.HERE.parent.parent / "include" / "fdtd.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(fdtd_\w+)\s*\(", text, flags=re.M)))


def test_exports_every_declared_symbol(engine_lib):
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(engine_lib, n), n
    assert set(names) == set(_lib.EXPORTED)


def test_argument_errors(engine_lib):
    with pytest.raises(ValueError):
        _lib.Simulation(1, 4, 4)
    sim = _lib.Simulation(4, 5, 6)
    with pytest.raises(ValueError, match="Expected shape on axis 2"):
        sim.set_coefficient("Ca_ex_y", np.zeros((4, 5, 7), np.float32))
    with pytest.raises(ValueError, match="Unknown coefficient"):
        sim.set_coefficient("Ca_xx", np.zeros((4, 5, 6), np.float32))
    with pytest.raises(_lib.FdtdError, match="Coefficient not set"):
        sim.compile()
    for name in COEFF_NAMES:
        sim.set_coefficient(name, np.ones((4, 5, 6), np.float32))
    sim.add_probe(2, (1, 1, 0))           # ez at x=1, y=1 -> cell (0, 0, 0)
    assert sim.compile()["n_rows"] >= 2
    sim.add_probe(0, (0, 0, 3))           # ex at y=0 lies on the PEC edge
    with pytest.raises(_lib.FdtdError, match="Source cannot be placed on grid edge"):
        sim.compile()
    # the pool trim checks its argument before it touches a device
    with pytest.raises(_lib.FdtdError, match="keep_bytes must be >= 0"):
        _lib.trim_memory(-1)


@pytest.fixture(scope="module")
def small():
    return mg.build_model(S.FDTD_Solver, geo.Box, geo.Rectangle, geo.Line, mg.grid_edges(),
                          lambda s, e: s.generate_mesh(grid=e))


def _table(s):
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)
    sim = _lib.Simulation(Nx, Ny, Nz)
    sim.set_coefficients(co)
    for p in pr:
        sim.add_probe(p["field"], p["idx"], p["is_source"], p["values"] if p["is_source"] else None)
    ids, rows = sim.material_table()
    return ids, rows, pr, Nt


def test_table_reproduces_coefficients(engine_lib, small):
    """Every non-boundary cell's row holds exactly the reference coefficients."""
    ids, rows, pr, Nt = _table(small)
    co = small.pack_inputs(gpu=True)[0]
    slot = dict(zip(COEFF_NAMES, [0, 2, 1, 3, 4, 6, 5, 7, 8, 10, 9, 11, 12, 15, 13, 14, 16, 17,
                                   18, 21, 19, 20, 22, 23, 24, 27, 25, 26, 28, 29]))
    inner = (slice(0, -1), slice(0, -1), slice(0, -1))
    for name, arr in co.items():
        got = rows[:, slot[name]].view(np.float32)[ids]
        assert np.array_equal(got[inner].view(np.uint32), arr[inner].view(np.uint32)), name
    assert rows[0].view(np.float32)[:30].tolist() == [0.0] * 30


def test_kernel_arithmetic_model_matches_oracle(engine_lib, oracle_lib, small):
    ids, rows, pr, Nt = _table(small)
    src = np.array([p["values"] for p in pr])
    rec = km.run_model(ids, rows, None, km.shifted_probes(pr), src, Nt)
    _, ref = run_oracle(small)
    assert rel_l2(rec, ref) < 1e-6


def test_kernel_arithmetic_model_edge_corrected(engine_lib, oracle_lib):
    """PEC edge corrections (H rows with Db1 != Db2 next to the trace edges,
    pinned to the reference by setup_edge.npz) through the material table."""
    s = mg.with_edge_corrections(mg.build_model(S.FDTD_Solver, geo.Box, geo.Rectangle, geo.Line, mg.grid_edges(),
                                                lambda m, e: m.generate_mesh(grid=e)))
    ids, rows, pr, Nt = _table(s)
    src = np.array([p["values"] for p in pr])
    rec = km.run_model(ids, rows, None, km.shifted_probes(pr), src, Nt)
    _, ref = run_oracle(s)
    assert rel_l2(rec, ref) < 1e-6


def test_component_split_flags(engine_lib):
    """Bit 8 + c of a row marks component c (ex ey ez hx hy hz) stored as its
    split pair: exactly where its two decays differ (or it carries a source)."""
    s = configs.microstrip(n=(24, 24, 20), n_pml=4, nt=10)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)
    sim = _lib.Simulation(Nx, Ny, Nz)
    sim.set_coefficients(co)
    ids, rows = sim.material_table()
    flags = rows[:, 30][ids]
    pairs = (("Ca_ex_y", "Ca_ex_z"), ("Ca_ey_z", "Ca_ey_x"), ("Ca_ez_x", "Ca_ez_y"),
             ("Da_hx_y", "Da_hx_z"), ("Da_hy_z", "Da_hy_x"), ("Da_hz_x", "Da_hz_y"))
    inner = (slice(0, -1), slice(0, -1), slice(0, -1))   # away from the zeroed / guarded planes
    for c, (a, b) in enumerate(pairs):
        split = (flags & (1 << (8 + c))) != 0
        assert np.array_equal(split[inner], (co[a] != co[b])[inner]), a
    # a cell of the z-PML slab away from the x and y slabs: ez and hz decay alike
    f = int(flags[Nx // 2, Ny // 2, 1])
    assert f & (1 << 8) and f & (1 << 9) and not f & (1 << 10)
    assert f & (1 << 11) and f & (1 << 12) and not f & (1 << 13)
    # the any-component bits follow
    assert np.array_equal((flags & 1) != 0, (flags & (7 << 8)) != 0)
    assert np.array_equal((flags & 2) != 0, (flags & (7 << 11)) != 0)


def test_split_flags_cover_pml(engine_lib):
    s = configs.microstrip(n=(24, 24, 20), n_pml=4, nt=10)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)
    sim = _lib.Simulation(Nx, Ny, Nz)
    sim.set_coefficients(co)
    ids, rows = sim.material_table()
    esplit = (rows[:, 30] & 1)[ids] != 0
    # cells where the two E splits of a component have different Ca must be split
    for a, b in (("Ca_ex_y", "Ca_ex_z"), ("Ca_ey_z", "Ca_ey_x"), ("Ca_ez_x", "Ca_ez_y")):
        diff = co[a] != co[b]
        diff[-1] = False          # x-max plane is zeroed (solver.cpp:294-311)
        diff[:, -1] = False       # guarded planes (solver.cu:152-185)
        diff[:, :, -1] = False
        assert not np.any(diff & ~esplit), a
    # the deep interior is unsplit
    assert not esplit[8:-8, 8:-8, 8:-8].any()


def test_borrowed_coefficients(engine_lib, small):
    """fdtd_set_coefficient_view lends the arrays: the same table as copies,
    and the box patch copies a borrowed array before writing to it."""
    co, pr, mo, mem, Nx, Ny, Nz, Nt = small.pack_inputs(gpu=True)
    a = _lib.Simulation(Nx, Ny, Nz)
    a.set_coefficients(co)
    lent = {k: v.copy() for k, v in co.items()}
    b = _lib.Simulation(Nx, Ny, Nz)
    b.set_coefficients(lent, borrow=True)
    ids_a, rows_a = a.material_table()
    ids_b, rows_b = b.material_table()
    assert np.array_equal(ids_a, ids_b) and np.array_equal(rows_a, rows_b)
    box = (4, 6, 5, 7, 3, 5)
    before = {k: v.copy() for k, v in lent.items()}
    b.set_box_coefficients(box, np.full((3, 3, 2, 2, 2), 0.5))
    for k in lent:
        assert np.array_equal(lent[k], before[k]), k
    ids_p, rows_p = b.material_table()
    x, y, z = 4, 5, 3
    assert rows_p[ids_p[x, y, z], 0].view(np.float32) == np.float32(0.5)
    a.close()
    b.close()


def test_table_limit_is_reported(engine_lib):
    """More distinct cell rows than the 16-bit material index addresses is an
    error of the compile, not a wrap-around."""
    rng = np.random.default_rng(0)
    shape = (42, 41, 40)            # 68,880 cells, each its own row
    sim = _lib.Simulation(*shape)
    for name in COEFF_NAMES:
        sim.set_coefficient(name, rng.uniform(0.5, 1.0, shape).astype(np.float32))
    with pytest.raises(_lib.FdtdError, match="at most 65536"):
        sim.compile()
    sim.close()


def test_split_storage_plan_confines_pml_pairs_to_the_slabs(engine_lib):
    """The split pairs of the PML live in slab stores of the PML's thickness
    (8 cells on every face here), and the only split cells outside them are
    the ports' soft-source cells, each on a table row of its own."""
    s = configs.boxes(n=(64, 56, 40), n_pml=8, n_boxes=6, nt=20, n_ports=2, n_probes=3)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)
    sim = _lib.Simulation(Nx, Ny, Nz)
    sim.set_coefficients(co)
    for p in pr:
        sim.add_probe(p["field"], p["idx"], p["is_source"], p["values"][:Nt] if p["is_source"] else None)
    sim.compile()
    st = sim.stats()
    ids, rows = sim.material_table()
    sim.close()
    assert st["split_slab"] == [8] * 6
    n = Nx * Ny * Nz
    assert st["slab_cells"] == n - (Nx - 16) * (Ny - 16) * (Nz - 16)
    split = ((rows[:, 30] & 3) != 0)[ids]
    inner = split[8:-8, 8:-8, 8:-8]
    assert st["sparse_split_cells"] == int(inner.sum()) > 0
    # the sparse cells are source cells; each has its own row
    inner_ids = ids[8:-8, 8:-8, 8:-8][inner]
    assert len(np.unique(inner_ids)) == len(inner_ids)
    assert ((rows[inner_ids, 30] >> 16) > 0).all()   # they carry probe entries (the port sources)


def test_sparse_split_cells_get_slots_in_cell_order(engine_lib):
    """Split cells inside the core box that carry no probe (here: interior
    cells given differing split decays) get rows of their own whose word 31
    numbers their sparse slots after the probe entries, in cell order."""
    s = configs.boxes(n=(64, 56, 40), n_pml=8, n_boxes=6, nt=20, n_ports=2, n_probes=3)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)
    co = {k: np.array(v) for k, v in co.items()}
    planted = [(20, 30, 15), (20, 30, 16), (20, 41, 9), (33, 12, 30), (47, 47, 31)]
    for c in planted:
        co["Ca_ex_z"][c] = np.float32(0.5) * co["Ca_ex_y"][c]
    sim = _lib.Simulation(Nx, Ny, Nz)
    sim.set_coefficients(co)
    for p in pr:
        sim.add_probe(p["field"], p["idx"], p["is_source"], p["values"][:Nt] if p["is_source"] else None)
    sim.compile()
    st = sim.stats()
    ids, rows = sim.material_table()
    sim.close()
    assert st["split_slab"] == [8] * 6
    split = ((rows[:, 30] & 3) != 0)[ids]
    inner = np.zeros_like(split)
    inner[8:-8, 8:-8, 8:-8] = split[8:-8, 8:-8, 8:-8]
    assert st["sparse_split_cells"] == int(inner.sum())
    slots = [int(rows[ids[c], 31]) for c in planted]   # planted in cell order
    n_probe_entries = len(pr)
    assert all(sl >= n_probe_entries for sl in slots)
    assert slots == sorted(slots) and len(set(slots)) == len(slots)
    assert all((rows[ids[c], 30] >> 16) == 0 for c in planted)   # no probe entries on them
