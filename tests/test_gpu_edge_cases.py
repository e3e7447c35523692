"""Edge cases of the engine on the GPU: tiny and ragged grids (smaller than
one tile, sizes that leave partial tiles in x, y and z), every cell a
distinct row with split components, a soft source and probes on the grid's
first and last cells, a run without probes, and a one-step run.

Random coefficients give every cell its own table row and most cells split
E and H components, so the streaming kernel's split paths (here one slab
store covers the grid), halo recomputation and zero-filled edges are all
exercised; it must give the plain kernel's bits exactly (the plain kernel's
parity with the oracle is tests/test_gpu_parity.py's). PML models with slabs
on all six faces and ragged x rows exercise the per-face stores, the two
staged regions of corner tiles and the sparse store of the port cells."""
import numpy as np
import pytest

from modelgen import configs
from rfnetwork_b200 import _lib
from rfnetwork_b200.solver_constants import COEFF_NAMES

pytestmark = pytest.mark.gpu


def _random_sim(shape, seed, nt, variant, probes=True, **kernel):
    rng = np.random.default_rng(seed)
    sim = _lib.Simulation(*shape)
    sim.set_kernel(variant, **kernel)
    for name in COEFF_NAMES:
        if name.startswith("Ca") or name.startswith("Da"):
            a = rng.uniform(0.9, 1.0, shape)
        else:
            a = rng.uniform(0.0, 0.1, shape) * rng.choice([-1.0, 1.0], shape)
        sim.set_coefficient(name, a.astype(np.float32))
    nx, ny, nz = shape
    if probes:
        t = np.arange(nt, dtype=np.float32)
        sim.add_probe(2, (nx // 2, ny // 2, nz // 2), True, np.sin(0.3 * t) * np.exp(-((t - 10) / 6) ** 2))
        # every field on the first and on the last cell the Yee shift allows
        for f in range(6):
            lo = [1 if f in (1, 2, 3) else 0, 1 if f in (0, 2, 4) else 0, 1 if f in (0, 1, 5) else 0]
            sim.add_probe(f, tuple(lo))
            sim.add_probe(f, (nx - 1, ny - 1, nz - 1))
    return sim


@pytest.mark.parametrize("shape", [(2, 2, 2), (3, 5, 2), (33, 9, 5), (40, 17, 3), (31, 8, 27), (64, 1 + 8, 64)])
def test_ragged_grids_stream_equals_plain(engine_lib, shape):
    nt = 40
    plain = _random_sim(shape, 1, nt, 0)
    plain.run(nt)
    ref = plain.probe_values()
    plain.close()
    assert np.isfinite(ref).all() and np.abs(ref).max() > 0
    for variant, ty, stages, zchunk in ((1, 8, 4, 0), (1, 4, 5, 1), (1, 6, 3, 2), (1, 8, 8, 3), (1, 12, 3, 1)):
        sim = _random_sim(shape, 1, nt, variant, tile_y=ty, stages=stages, zchunk=zchunk)
        sim.run(nt)
        got = sim.probe_values()
        sim.close()
        assert np.array_equal(got, ref), (shape, variant, ty, stages, zchunk)


def test_run_without_probes_and_one_step(engine_lib):
    sim = _random_sim((20, 12, 10), 2, 5, 1, probes=False)
    sim.run(5)                      # no probes: nothing recorded, nothing to read
    assert sim.stats()["step_launches"] == 5
    sim.close()
    a = _random_sim((20, 12, 10), 3, 1, 0)
    b = _random_sim((20, 12, 10), 3, 1, 1)
    a.run(1)
    b.run(1)
    assert np.array_equal(a.probe_values(), b.probe_values())
    a.close()
    b.close()


@pytest.mark.parametrize("kernel", [(1, 8, 4, 0), (1, 4, 6, 2)])
def test_batch_of_tiny_grids_equals_single_runs(engine_lib, kernel):
    """A batch whose members are smaller than one tile or leave ragged tiles
    gives each member the bits of its own run."""
    shapes = [(2, 2, 2), (3, 5, 2), (33, 9, 5), (40, 17, 3), (31, 8, 27)]
    nt = 30
    singles = []
    for k, shape in enumerate(shapes):
        sim = _random_sim(shape, 10 + k, nt, 1, tile_y=8, stages=4, zchunk=0)
        sim.run(nt)
        singles.append(sim.probe_values())
        sim.close()
    sims = [_random_sim(shape, 10 + k, nt, 1) for k, shape in enumerate(shapes)]
    batch = _lib.Batch(sims)
    batch.set_kernel(*kernel)
    batch.run(nt)
    for sim, ref in zip(sims, singles):
        assert np.array_equal(sim.probe_values(), ref)
    batch.close()
    for sim in sims:
        sim.close()


def _boxes_sim(shape, nt, kernel):
    m = configs.boxes(n=shape, n_pml=8, n_boxes=6, nt=nt, n_ports=2, n_probes=4)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = m.pack_inputs(gpu=True)
    sim = _lib.Simulation(Nx, Ny, Nz)
    sim.set_kernel(*kernel)
    sim.set_coefficients(co)
    for q in pr:
        sim.add_probe(q["field"], q["idx"], q["is_source"], q["values"][:Nt] if q["is_source"] else None)
    return sim, len(pr)


@pytest.mark.parametrize("shape", [(64, 56, 40), (70, 60, 37)])
def test_slab_stores_stream_equals_plain(engine_lib, shape):
    """8-cell PML on all faces: the split pairs live in six slab stores (and a
    sparse store for the port cells); every streaming shape gives the plain
    kernel's bits, and the stores hold 96 bytes per slab cell and per sparse
    slot, nothing for the core."""
    nt = 60
    sim, n_probes = _boxes_sim(shape, nt, (0, 0, 4, 0))
    sim.run(nt)
    ref = sim.probe_values()
    st = sim.stats()
    sim.close()
    assert np.isfinite(ref).all() and np.abs(ref).max() > 0
    assert st["split_slab"] == [8] * 6
    nx, ny, nz = shape
    pitch = (nx + 31) // 32 * 32
    # z and y stores span the pitch; x stores an even number of pairs from an
    # even origin over the core rows
    oxh = (nx - 8) // 2 * 2
    x_width = 8 + (nx - oxh + 1) // 2 * 2
    slab_cells = 2 * 8 * ny * pitch + 2 * 8 * (nz - 16) * pitch + x_width * (ny - 16) * (nz - 16)
    # sparse slots: one per probe-list entry (a probe cell's slot) and per other split cell
    slots, rest = divmod(st["split_bytes"] - 96 * slab_cells, 96)
    assert rest == 0
    assert st["sparse_split_cells"] <= slots <= st["sparse_split_cells"] + n_probes
    for kernel in ((1, 8, 6, 0), (1, 8, 4, 5), (1, 4, 6, 0), (1, 6, 3, 2), (1, 12, 3, 0)):
        sim, _ = _boxes_sim(shape, nt, kernel)
        sim.run(nt)
        got = sim.probe_values()
        sim.close()
        assert np.array_equal(got, ref), kernel


def test_autotuner_cost_in_stats(engine_lib):
    # a grid size no other test uses, so the first engine tunes and the second
    # takes the cached shape
    shape = (45, 23, 19)
    first = _random_sim(shape, 5, 12, 1, tile_y=0)
    first.run(12)
    st = first.stats()
    ref = first.probe_values()
    first.close()
    assert st["tune_trials"] >= 2 and st["tune_ms"] > 0.0
    second = _random_sim(shape, 5, 12, 1, tile_y=0)
    second.run(12)
    st2 = second.stats()
    got = second.probe_values()
    second.close()
    assert st2["tune_trials"] == 0 and st2["tune_ms"] == 0.0
    assert (st2["tile_y"], st2["stages"], st2["zchunk"]) == (st["tile_y"], st["stages"], st["zchunk"])
    # the trial steps leave no trace in the results
    assert np.array_equal(got, ref)


def test_trim_memory_returns_pooled_memory(engine_lib):
    s = configs.microstrip(n=(128, 96, 64), n_pml=6, nt=8)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)

    def make():
        sim = _lib.Simulation(Nx, Ny, Nz)
        sim.set_coefficients(co)
        for p in pr:
            sim.add_probe(p["field"], p["idx"], p["is_source"], p["values"][:Nt] if p["is_source"] else None)
        return sim

    sim = make()
    sim.run(Nt)
    ref = sim.probe_values()
    sim.close()
    before = _lib.trim_memory(1 << 60)  # keeps every unused byte: only reads the pool
    after = _lib.trim_memory(0)
    fields = 12 * Nx * Ny * Nz * 4
    assert before["reserved"] - after["reserved"] >= fields // 2
    assert after["used"] == before["used"] and after["reserved"] >= after["used"]
    # the engine allocates again from the trimmed pool
    again = make()
    again.run(Nt)
    assert np.array_equal(again.probe_values(), ref)
    again.close()
    with pytest.raises(_lib.FdtdError):
        _lib.trim_memory(-1)
