"""fdtd_step_noalloc: stepping a grid held in caller-owned device buffers.

The entry point exists for callers that cannot let a library allocate device
memory. A framework whose caching allocator owns the GPU memory, or a service
with a fixed memory budget, needs every byte to come from its own pool; a
cudaMalloc would escape that accounting, and a cudaFree waits for the whole
device. The test plays such a caller: torch allocates every buffer, the
entry point allocates nothing (device memory in use and torch's reserved
pool are unchanged across a call), and two calls in a row must reproduce, bit
for bit, what the ordinary entry point (fdtd_run, with the same plain step
kernel) records for the same model.

This file is collected last, so a run that stops at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

import kernel_model as km
from helpers import rel_l2
from modelgen import configs
from rfnetwork_b200 import _lib

TOL = 1e-5


class DeviceGrid(ctypes.Structure):
    """fdtd_device_grid of include/fdtd.h."""
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("pitch", ctypes.c_int),
        ("nt", ctypes.c_int),
        ("fields", ctypes.c_void_p), ("splits", ctypes.c_void_p), ("mat", ctypes.c_void_p),
        ("rows", ctypes.c_void_p), ("cell_probes", ctypes.c_void_p), ("src", ctypes.c_void_p),
        ("rec", ctypes.c_void_p), ("is_src", ctypes.c_void_p),
        ("n_rows", ctypes.c_int), ("n_probes", ctypes.c_int),
    ]


def _entry(lib):
    fn = lib.fdtd_step_noalloc
    fn.argtypes = [ctypes.POINTER(DeviceGrid), ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return fn


def _cell_probes(probe_dicts, ny, nz):
    """(probe, field) pairs grouped by shifted cell, ties in probe order (the layout the rows index)."""
    shifted = km.shifted_probes(probe_dicts)
    keyed = [((x * ny + y) * nz + z, p, f) for p, (f, x, y, z, _) in enumerate(shifted)]
    keyed.sort(key=lambda t: t[0])  # stable: equal cells keep probe order
    return np.array([[p, f] for _, p, f in keyed], dtype=np.int32).reshape(-1)


def test_rejects_bad_sizes_without_touching_the_gpu(engine_lib):
    fn = _entry(engine_lib)
    g = DeviceGrid(nx=4000, ny=4000, nz=8, pitch=4000, nt=10, n_rows=1)
    assert fn(ctypes.byref(g), 0, 1, None) == 4           # FDTD_ERR_LIMIT: tile list over capacity
    assert b"tiles" in engine_lib.fdtd_global_error()
    g = DeviceGrid(nx=16, ny=16, nz=8, pitch=16, nt=10, n_rows=1)
    assert fn(ctypes.byref(g), 0, 1, None) == 1           # FDTD_ERR_ARG: no buffers
    assert fn(ctypes.byref(g), 5, 6, None) == 1           # steps beyond nt
    g.pitch = 8
    assert fn(ctypes.byref(g), 0, 1, None) == 1           # pitch < nx
    g = DeviceGrid(nx=16, ny=16, nz=8, pitch=32, nt=10, n_rows=0)
    assert fn(ctypes.byref(g), 0, 1, None) == 1           # no material rows
    assert b"n_rows" in engine_lib.fdtd_global_error()
    g.n_rows, g.n_probes = 70000, 0
    assert fn(ctypes.byref(g), 0, 1, None) == 1           # more rows than a 16-bit index addresses


@pytest.mark.gpu
def test_two_calls_match_fdtd_run(engine_lib):
    import torch

    fn = _entry(engine_lib)
    s = configs.microstrip(n=(40, 30, 26), n_pml=4, nt=160)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)

    # the existing entry point on the same model, with the same (plain) step kernel
    sim = _lib.Simulation(Nx, Ny, Nz)
    sim.set_kernel(0)
    sim.set_coefficients(co)
    for p in pr:
        sim.add_probe(p["field"], p["idx"], p["is_source"], p["values"][:Nt] if p["is_source"] else None)
    sim.run(Nt)
    ref = sim.probe_values()
    ids, rows = sim.material_table()
    sim.close()
    assert np.abs(ref).max() > 0

    # caller-owned device buffers, allocated by torch (not by the library)
    dev = torch.device("cuda", 0)
    pitch = (Nx + 31) // 32 * 32
    N = Nz * Ny * pitch
    mat = np.zeros((Nz, Ny, pitch), np.uint16)
    mat[:, :, :Nx] = ids.transpose(2, 1, 0)
    P = len(pr)
    src = np.zeros((P, Nt), np.float32)
    is_src = np.zeros(P, np.int32)
    for i, p in enumerate(pr):
        if p["is_source"]:
            src[i] = p["values"][:Nt]
            is_src[i] = 1
    t = {
        "fields": torch.zeros(12 * N, dtype=torch.float32, device=dev),
        "splits": torch.zeros(24 * N, dtype=torch.float32, device=dev),
        "mat": torch.from_numpy(mat.reshape(-1).view(np.int16)).to(dev),
        "rows": torch.from_numpy(rows.reshape(-1).view(np.int32)).to(dev),
        "cell_probes": torch.from_numpy(_cell_probes(pr, Ny, Nz)).to(dev),
        "src": torch.from_numpy(src.reshape(-1)).to(dev),
        "rec": torch.zeros(P * Nt, dtype=torch.float32, device=dev),
        "is_src": torch.from_numpy(is_src).to(dev),
    }
    g = DeviceGrid(nx=Nx, ny=Ny, nz=Nz, pitch=pitch, nt=Nt, n_rows=rows.shape[0], n_probes=P,
                   **{k: v.data_ptr() for k, v in t.items()})
    stream = torch.cuda.current_stream(dev).cuda_stream

    def memory():
        torch.cuda.synchronize(dev)
        free, total = torch.cuda.mem_get_info(dev)
        return total - free, torch.cuda.memory_reserved(dev)

    half = Nt // 2
    # first call: steps 0 .. half-1 (its set-up may load the library's kernels)
    assert fn(ctypes.byref(g), 0, half, ctypes.c_void_p(stream)) == 0, engine_lib.fdtd_global_error()
    torch.cuda.synchronize(dev)
    rec = t["rec"].cpu().numpy().reshape(P, Nt)
    np.testing.assert_array_equal(rec[:, :half], ref[:, :half])
    assert not rec[:, half:].any()
    # second call continues the same grid: steps half .. Nt-1, allocating nothing
    before = memory()
    assert fn(ctypes.byref(g), half, Nt - half, ctypes.c_void_p(stream)) == 0, engine_lib.fdtd_global_error()
    after = memory()
    assert after == before, f"device memory in use / torch reserved changed: {before} -> {after}"
    rec = t["rec"].cpu().numpy().reshape(P, Nt)
    np.testing.assert_array_equal(rec, ref)
    assert rel_l2(rec, ref) <= TOL
    assert np.isfinite(rec).all()
