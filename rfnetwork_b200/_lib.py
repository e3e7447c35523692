"""ctypes binding of librfn_fdtd.so (declarations: include/fdtd.h).

The library is the only compute path: if it is missing or cannot be loaded,
every entry point raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "librfn_fdtd.so"

FDTD_ERRORS = {1: "invalid argument", 2: "CUDA error", 3: "call out of order", 4: "size limit", 5: "device error",
               6: "non-finite result"}

EXPORTED = (
    "fdtd_create", "fdtd_set_coefficient", "fdtd_add_probe", "fdtd_add_monitor", "fdtd_set_dft",
    "fdtd_compile", "fdtd_get_material_table",
    "fdtd_run", "fdtd_run_async", "fdtd_synchronize", "fdtd_set_stream", "fdtd_get_probe_values",
    "fdtd_set_kernel", "fdtd_batch_set_kernel", "fdtd_set_coefficient_view",
    "fdtd_get_dft", "fdtd_get_monitor", "fdtd_get_stats", "fdtd_last_error", "fdtd_destroy",
    "fdtd_batch_create", "fdtd_batch_run", "fdtd_batch_set_stream", "fdtd_batch_get_stats",
    "fdtd_batch_last_error", "fdtd_batch_destroy", "fdtd_global_error", "fdtd_step_noalloc",
    "fdtd_run_checkpointed", "fdtd_run_recorded", "fdtd_adjoint", "fdtd_batch_run_recorded",
    "fdtd_batch_run_checkpointed", "fdtd_batch_adjoint", "fdtd_set_graph", "fdtd_set_box_coefficients", "fdtd_nf2ff", "fdtd_set_debug",
    "fdtd_trim_memory",
)


class Nf2ffFace(ctypes.Structure):
    _fields_ = [("axis", ctypes.c_int), ("n0", ctypes.c_int), ("n1", ctypes.c_int), ("pos", ctypes.c_float),
                ("r0", ctypes.c_void_p), ("r1", ctypes.c_void_p), ("ds", ctypes.c_void_p), ("J", ctypes.c_void_p),
                ("M", ctypes.c_void_p)]


class FdtdStats(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("nt", ctypes.c_int),
        ("n_rows", ctypes.c_int), ("id_bytes", ctypes.c_int),
        ("e_split_cells", ctypes.c_int64), ("h_split_cells", ctypes.c_int64),
        ("n_tiles", ctypes.c_int), ("step_launches", ctypes.c_int64), ("dft_launches", ctypes.c_int64),
        ("last_run_ms", ctypes.c_double), ("compile_ms", ctypes.c_double),
        ("variant", ctypes.c_int), ("tile_y", ctypes.c_int), ("stages", ctypes.c_int), ("zchunk", ctypes.c_int),
        ("grid", ctypes.c_int), ("h2d_bytes", ctypes.c_int64), ("d2h_bytes", ctypes.c_int64),
        ("adjoint_launches", ctypes.c_int64), ("adjoint_ms", ctypes.c_double),
        ("split_slab", ctypes.c_int * 6), ("slab_cells", ctypes.c_int64), ("sparse_split_cells", ctypes.c_int64),
        ("split_bytes", ctypes.c_int64), ("tune_ms", ctypes.c_double), ("tune_trials", ctypes.c_int),
    ]

    def as_dict(self):
        return {k: (list(getattr(self, k)) if k == "split_slab" else getattr(self, k)) for k, _ in self._fields_}



_lib = None


def load():
    """Load the engine library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH.name} is not built; run `python -m rfnetwork_b200.build` "
                           "(the FDTD engine has no CPU fallback).")
    lib = ctypes.CDLL(str(LIB_PATH))
    vp, ip, i64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64
    pp = ctypes.POINTER(ctypes.c_void_p)
    sig = {
        "fdtd_create": ([ip, ip, ip, pp], ip),
        "fdtd_set_coefficient": ([vp, ctypes.c_char_p, vp, ip, ip, ip], ip),
        "fdtd_set_coefficient_view": ([vp, ctypes.c_char_p, vp, ip, ip, ip], ip),
        "fdtd_add_probe": ([vp, ip, ip, ip, ip, ip, vp, ip, ctypes.POINTER(ip)], ip),
        "fdtd_add_monitor": ([vp, ip, ip, ip, ip, ip, vp, ip, ctypes.POINTER(ip)], ip),
        "fdtd_set_dft": ([vp, ip, ip, vp, vp, vp, ip, vp], ip),
        "fdtd_compile": ([vp, ctypes.POINTER(ip), ctypes.POINTER(i64), ctypes.POINTER(i64)], ip),
        "fdtd_get_material_table": ([vp, vp, i64, vp, ip], ip),
        "fdtd_set_kernel": ([vp, ip, ip, ip, ip], ip),
        "fdtd_batch_set_kernel": ([vp, ip, ip, ip, ip], ip),
        "fdtd_run": ([vp, ip], ip),
        "fdtd_run_async": ([vp, ip], ip),
        "fdtd_synchronize": ([vp], ip),
        "fdtd_set_stream": ([vp, vp], ip),
        "fdtd_set_graph": ([vp, ip], ip),
        "fdtd_set_debug": ([vp, ctypes.c_uint, ip], ip),
        "fdtd_set_box_coefficients": ([vp, vp, vp], ip),
        "fdtd_nf2ff": ([vp, ip, ip, vp, ip, vp, ip, vp, vp], ip),
        "fdtd_get_probe_values": ([vp, vp, ip, ip], ip),
        "fdtd_get_dft": ([vp, vp, ip, ip], ip),
        "fdtd_get_monitor": ([vp, ip, vp, i64], ip),
        "fdtd_get_stats": ([vp, ctypes.POINTER(FdtdStats)], ip),
        "fdtd_last_error": ([vp], ctypes.c_char_p),
        "fdtd_destroy": ([vp], None),
        "fdtd_batch_create": ([pp, ip, pp], ip),
        "fdtd_batch_run": ([vp, ip], ip),
        "fdtd_batch_set_stream": ([vp, vp], ip),
        "fdtd_batch_get_stats": ([vp, ctypes.POINTER(FdtdStats)], ip),
        "fdtd_batch_last_error": ([vp], ctypes.c_char_p),
        "fdtd_batch_destroy": ([vp], None),
        "fdtd_global_error": ([], ctypes.c_char_p),
        "fdtd_trim_memory": ([i64, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)], ip),
        "fdtd_run_checkpointed": ([vp, ip, ip], ip),
        "fdtd_run_recorded": ([vp, ip, vp], ip),
        "fdtd_adjoint": ([vp, vp, ip, ip, vp, vp], ip),
        "fdtd_batch_run_recorded": ([vp, ip, vp], ip),
        "fdtd_batch_run_checkpointed": ([vp, ip, ip, vp], ip),
        "fdtd_batch_adjoint": ([vp, pp, pp], ip),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def _ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


class FdtdError(RuntimeError):
    """An engine call failed; ``code`` is its FDTD_ERR_* status (include/fdtd.h)."""

    def __init__(self, msg: str, code: int = 0):
        super().__init__(msg)
        self.code = code


def _dj_pairs(dJ_dX) -> np.ndarray:
    """complex [series, freq] -> float64 [series, freq, (re, im)]."""
    return np.ascontiguousarray(np.stack([np.real(dJ_dX), np.imag(dJ_dX)], axis=-1), dtype=np.float64)


def _grad_shape(b) -> tuple:
    return (3, 3, int(b[1] - b[0]), int(b[3] - b[2]), int(b[5] - b[4]))


class Simulation:
    """One FDTD grid on the GPU (an ``fdtd_sim`` handle).

    Coefficients are the reference's GPU-shaped (nx, ny, nz) float32 arrays.
    """

    def __init__(self, nx: int, ny: int, nz: int):
        self.lib = load()
        h = ctypes.c_void_p()
        rc = self.lib.fdtd_create(int(nx), int(ny), int(nz), ctypes.byref(h))
        if rc:
            raise ValueError(self.lib.fdtd_global_error().decode())
        self.h = h
        self.shape = (int(nx), int(ny), int(nz))
        self.n_probes = 0
        self.n_series = 0
        self.n_freq = 0
        self.monitors = []
        self.nt = None
        self._borrowed = {}   # arrays lent to the engine by set_coefficient(borrow=True)

    def _check(self, rc):
        if rc:
            msg = self.lib.fdtd_last_error(self.h).decode()
            if rc == 1:
                raise ValueError(msg)
            raise FdtdError(f"{FDTD_ERRORS.get(rc, rc)}: {msg}", rc)

    def set_coefficient(self, name: str, arr: np.ndarray, borrow: bool = False):
        """Copy the array into the engine, or with ``borrow`` lend it (no copy):
        the simulation then keeps a reference to it until it is closed."""
        a = np.ascontiguousarray(arr, dtype=np.float32)
        if a.ndim != 3:
            raise ValueError("Invalid data array. Wrong number of dimensions.")
        if borrow:
            self._check(self.lib.fdtd_set_coefficient_view(self.h, name.encode(), _ptr(a), *a.shape))
            self._borrowed[name] = a
        else:
            self._check(self.lib.fdtd_set_coefficient(self.h, name.encode(), _ptr(a), *a.shape))
            self._borrowed.pop(name, None)

    def set_coefficients(self, coefficients: dict, borrow: bool = False):
        for k, v in coefficients.items():
            self.set_coefficient(k, v, borrow)

    def add_probe(self, field: int, idx, is_source: bool = False, values=None) -> int:
        out = ctypes.c_int()
        if values is not None:
            v = np.ascontiguousarray(values, dtype=np.float32)
            rc = self.lib.fdtd_add_probe(self.h, int(field), int(idx[0]), int(idx[1]), int(idx[2]),
                                         int(bool(is_source)), _ptr(v), int(v.size), ctypes.byref(out))
        else:
            rc = self.lib.fdtd_add_probe(self.h, int(field), int(idx[0]), int(idx[1]), int(idx[2]),
                                         int(bool(is_source)), None, 0, ctypes.byref(out))
        self._check(rc)
        self.n_probes = out.value + 1
        return out.value

    def add_monitor(self, field: int, axis: int, position: int, n_step: int = 1, phase=None) -> int:
        out = ctypes.c_int()
        if phase is not None:
            ph = np.ascontiguousarray(phase, dtype=np.complex64)
            rc = self.lib.fdtd_add_monitor(self.h, int(field), int(axis), int(position), int(n_step),
                                           int(ph.shape[1]), _ptr(ph), int(ph.shape[0]), ctypes.byref(out))
            nf = int(ph.shape[1])
        else:
            rc = self.lib.fdtd_add_monitor(self.h, int(field), int(axis), int(position), int(n_step), 0, None, 0,
                                           ctypes.byref(out))
            nf = 0
        self._check(rc)
        nx, ny, nz = self.shape
        n1 = ny if axis == 0 else nx
        n2 = ny if axis == 2 else nz
        self.monitors.append(dict(n_freq=nf, n_step=int(n_step), n1=n1, n2=n2))
        return out.value

    def set_dft(self, terms, omega):
        """terms: iterable of (series, probe, weight); omega: radians per time step."""
        terms = list(terms)
        ts = np.array([t[0] for t in terms], dtype=np.int32)
        tp = np.array([t[1] for t in terms], dtype=np.int32)
        tw = np.array([t[2] for t in terms], dtype=np.float64)
        om = np.ascontiguousarray(omega, dtype=np.float64)
        n_series = int(ts.max()) + 1 if ts.size else 0
        self._check(self.lib.fdtd_set_dft(self.h, n_series, int(ts.size), _ptr(ts), _ptr(tp), _ptr(tw),
                                          int(om.size), _ptr(om)))
        self.n_series, self.n_freq = n_series, int(om.size)

    def compile(self) -> dict:
        """Build the material table on the host (no GPU needed)."""
        n = ctypes.c_int()
        e = ctypes.c_int64()
        h = ctypes.c_int64()
        self._check(self.lib.fdtd_compile(self.h, ctypes.byref(n), ctypes.byref(e), ctypes.byref(h)))
        return dict(n_rows=n.value, e_split_cells=e.value, h_split_cells=h.value)

    def material_table(self):
        """(ids [nx, ny, nz] uint16, rows [n_rows, 32] uint32) of the compiled table."""
        info = self.compile()
        ids = np.empty(self.shape, dtype=np.uint16)
        rows = np.empty((info["n_rows"], 32), dtype=np.uint32)
        self._check(self.lib.fdtd_get_material_table(self.h, _ptr(ids), int(ids.size), _ptr(rows),
                                                     info["n_rows"]))
        return ids, rows

    def set_kernel(self, variant: int = 1, tile_y: int = 0, stages: int = 4, zchunk: int = 0):
        """Pick the step kernel (0 plain loads, 1 TMA streaming) and its tile shape (tile_y 0: autotuned)."""
        self._check(self.lib.fdtd_set_kernel(self.h, int(variant), int(tile_y), int(stages), int(zchunk)))

    def set_stream(self, stream_ptr: int):
        self._check(self.lib.fdtd_set_stream(self.h, ctypes.c_void_p(int(stream_ptr))))

    def set_graph(self, enabled: bool):
        """Replay the time loop as a CUDA graph (default) or launch every step from the host."""
        self._check(self.lib.fdtd_set_graph(self.h, int(bool(enabled))))

    def set_debug(self, wait_limit: int = 0, withhold_plane: int = -1):
        """Failure-path testing of the streaming kernel: pipeline waits give up
        after ``wait_limit`` polls (0: the default, about 2 s) and, with
        ``withhold_plane`` >= 0, that plane's loads are never issued."""
        self._check(self.lib.fdtd_set_debug(self.h, int(wait_limit), int(withhold_plane)))

    def run(self, nt: int):
        self.nt = int(nt)  # the records of a failed run stay readable
        self._check(self.lib.fdtd_run(self.h, int(nt)))

    def run_checkpointed(self, nt: int, every: int):
        """Run like ``run`` and keep a field snapshot every ``every`` steps for ``adjoint``."""
        self._check(self.lib.fdtd_run_checkpointed(self.h, int(nt), int(every)))
        self.nt = int(nt)

    def set_box_coefficients(self, box, coefs: np.ndarray):
        """E-update coefficients [3 components, (Ca, Cb1, Cb2), *box shape] of the cells of ``box``."""
        b = np.ascontiguousarray(box, dtype=np.int32)
        c = np.ascontiguousarray(coefs, dtype=np.float32)
        if c.shape != _grad_shape(b):
            raise ValueError(f"coefficients of shape {_grad_shape(b)} expected, got {c.shape}")
        self._check(self.lib.fdtd_set_box_coefficients(self.h, _ptr(b), _ptr(c)))

    def run_recorded(self, nt: int, box):
        """Run like ``run`` and record the forward history of ``box`` at every step for ``adjoint``."""
        b = np.ascontiguousarray(box, dtype=np.int32)
        self._check(self.lib.fdtd_run_recorded(self.h, int(nt), _ptr(b)))
        self.nt = int(nt)

    def adjoint(self, dJ_dX: np.ndarray, box) -> np.ndarray:
        """Gradient [3 components, (Ca, Cb1, Cb2), *box shape] of J given dJ/dX of the device DFT.

        dJ_dX: complex [n_series, n_freq] (dJ/dRe X + i dJ/dIm X); box: (x0, x1, y0, y1, z0, z1)."""
        g = _dj_pairs(dJ_dX)
        b = np.ascontiguousarray(box, dtype=np.int32)
        out = np.empty(_grad_shape(b), dtype=np.float64)
        self._check(self.lib.fdtd_adjoint(self.h, _ptr(g), g.shape[0], g.shape[1], _ptr(b), _ptr(out)))
        return out

    def run_async(self, nt: int):
        self._check(self.lib.fdtd_run_async(self.h, int(nt)))
        self.nt = int(nt)

    def synchronize(self):
        self._check(self.lib.fdtd_synchronize(self.h))

    def probe_values(self) -> np.ndarray:
        out = np.empty((self.n_probes, self.nt), dtype=np.float32)
        self._check(self.lib.fdtd_get_probe_values(self.h, _ptr(out), self.n_probes, self.nt))
        return out

    def dft(self) -> np.ndarray:
        out = np.empty((self.n_series, self.n_freq, 2), dtype=np.float64)
        self._check(self.lib.fdtd_get_dft(self.h, _ptr(out), self.n_series, self.n_freq))
        return out[..., 0] + 1j * out[..., 1]

    def monitor(self, m: int) -> np.ndarray:
        info = self.monitors[m]
        if info["n_freq"]:
            out = np.empty((info["n_freq"], info["n1"], info["n2"]), dtype=np.complex64)
        else:
            out = np.empty((self.nt // info["n_step"] + 1, info["n1"], info["n2"]), dtype=np.float32)
        self._check(self.lib.fdtd_get_monitor(self.h, int(m), _ptr(out), int(out.nbytes)))
        return out

    def stats(self) -> dict:
        st = FdtdStats()
        self._check(self.lib.fdtd_get_stats(self.h, ctypes.byref(st)))
        return st.as_dict()

    def close(self):
        if getattr(self, "h", None):
            self.lib.fdtd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Several simulations stepped together by one kernel launch per step."""

    def __init__(self, sims):
        self.lib = load()
        self.sims = list(sims)
        arr = (ctypes.c_void_p * len(self.sims))(*[s.h.value for s in self.sims])
        h = ctypes.c_void_p()
        rc = self.lib.fdtd_batch_create(arr, len(self.sims), ctypes.byref(h))
        if rc:
            raise ValueError(self.lib.fdtd_global_error().decode())
        self.h = h

    def run(self, nt: int):
        rc = self.lib.fdtd_batch_run(self.h, int(nt))
        if rc:
            raise FdtdError(f"{FDTD_ERRORS.get(rc, rc)}: {self.lib.fdtd_batch_last_error(self.h).decode()}")
        for s in self.sims:
            s.nt = int(nt)

    def _check(self, rc):
        if rc:
            msg = self.lib.fdtd_batch_last_error(self.h).decode()
            if rc == 1:
                raise ValueError(msg)
            raise FdtdError(f"{FDTD_ERRORS.get(rc, rc)}: {msg}", rc)

    def run_recorded(self, nt: int, boxes):
        """Batched ``Simulation.run_recorded``: boxes[i] is member i's gradient box."""
        b = np.ascontiguousarray(boxes, dtype=np.int32).reshape(len(self.sims), 6)
        self._check(self.lib.fdtd_batch_run_recorded(self.h, int(nt), _ptr(b)))
        self.boxes = b.copy()
        for s in self.sims:
            s.nt = int(nt)

    def run_checkpointed(self, nt: int, every: int, boxes):
        """Batched ``Simulation.run_checkpointed`` (state snapshots every ``every``
        steps); boxes[i] is member i's gradient box, fixed at the run."""
        b = np.ascontiguousarray(boxes, dtype=np.int32).reshape(len(self.sims), 6)
        self._check(self.lib.fdtd_batch_run_checkpointed(self.h, int(nt), int(every), _ptr(b)))
        self.boxes = b.copy()
        for s in self.sims:
            s.nt = int(nt)

    def adjoint(self, dJ_dX) -> list:
        """Gradients of all members after ``run_recorded`` or ``run_checkpointed``:
        dJ_dX[i] complex [series, freq] of member i."""
        gs = [_dj_pairs(d) for d in dJ_dX]
        outs = [np.empty(_grad_shape(b), dtype=np.float64) for b in self.boxes]
        n = len(self.sims)
        din = (ctypes.c_void_p * n)(*[g.ctypes.data for g in gs])
        dout = (ctypes.c_void_p * n)(*[o.ctypes.data for o in outs])
        self._check(self.lib.fdtd_batch_adjoint(self.h, din, dout))
        return outs

    def set_kernel(self, variant: int = 1, tile_y: int = 0, stages: int = 4, zchunk: int = 0):
        rc = self.lib.fdtd_batch_set_kernel(self.h, int(variant), int(tile_y), int(stages), int(zchunk))
        if rc:
            raise ValueError(self.lib.fdtd_batch_last_error(self.h).decode())

    def set_stream(self, stream_ptr: int):
        self.lib.fdtd_batch_set_stream(self.h, ctypes.c_void_p(int(stream_ptr)))

    def stats(self) -> dict:
        st = FdtdStats()
        self.lib.fdtd_batch_get_stats(self.h, ctypes.byref(st))
        return st.as_dict()

    def close(self):
        if getattr(self, "h", None):
            self.lib.fdtd_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def nf2ff(J_xyz, M_xyz, r_grid, ds_grid, surf_pos, ff_data) -> int:
    """Far-field transform with the arguments of the reference's core_func.nf2ff
    (rfnetwork/solver.py:3014, rfnetwork/core/src/postprocess.cpp:130-505).

    J_xyz[axis][side], M_xyz[axis][side]: complex64 [3, n_freq, n0, n1] surface
    currents; r_grid[axis][0/1]: float32 [n0, n1] cell centers (m) along the two
    other axes; ds_grid[axis]: [n0, n1] cell areas; surf_pos[axis][side]: face
    position (m); ff_data: dict with float32 beta, theta, phi (radians) and the
    complex64 [2, n_freq, n_theta, n_phi] array "data", written in place."""
    lib = load()
    keep, faces = [], []
    beta = np.ascontiguousarray(ff_data["beta"], dtype=np.float32)
    theta = np.ascontiguousarray(ff_data["theta"], dtype=np.float32)
    phi = np.ascontiguousarray(ff_data["phi"], dtype=np.float32)
    data = ff_data["data"]
    F = len(beta)
    if data.dtype != np.complex64 or data.shape != (2, F, len(theta), len(phi)) or not data.flags["C_CONTIGUOUS"]:
        raise ValueError("Invalid far-field data array. Expected complex64 (2, frequency, theta, phi).")
    for axis in range(3):
        r0 = np.ascontiguousarray(r_grid[axis][0], dtype=np.float32)
        r1 = np.ascontiguousarray(r_grid[axis][1], dtype=np.float32)
        ds = np.ascontiguousarray(np.real(ds_grid[axis]), dtype=np.float32)
        n0, n1 = ds.shape
        for side in range(2):
            J = np.ascontiguousarray(J_xyz[axis][side], dtype=np.complex64)
            M = np.ascontiguousarray(M_xyz[axis][side], dtype=np.complex64)
            if J.shape != (3, F, n0, n1) or M.shape != (3, F, n0, n1):
                raise ValueError("Invalid current array shape.")
            keep += [r0, r1, ds, J, M]
            faces.append(Nf2ffFace(axis, n0, n1, float(surf_pos[axis][side]), r0.ctypes.data, r1.ctypes.data,
                                   ds.ctypes.data, J.ctypes.data, M.ctypes.data))
    arr = (Nf2ffFace * len(faces))(*faces)
    rc = lib.fdtd_nf2ff(arr, len(faces), F, _ptr(beta), len(theta), _ptr(theta), len(phi), _ptr(phi), _ptr(data))
    if rc:
        raise FdtdError(f"{FDTD_ERRORS.get(rc, rc)}: {lib.fdtd_global_error().decode()}")
    return 0


def trim_memory(keep_bytes: int = 0) -> dict:
    """Return the engine's unused pooled device memory (current device) to the
    driver, keeping at most ``keep_bytes`` of unused reserve; returns the pool's
    reserved and in-use bytes afterwards."""
    lib = load()
    reserved, used = ctypes.c_int64(0), ctypes.c_int64(0)
    rc = lib.fdtd_trim_memory(int(keep_bytes), ctypes.byref(reserved), ctypes.byref(used))
    if rc:
        raise FdtdError(f"{FDTD_ERRORS.get(rc, rc)}: {lib.fdtd_global_error().decode()}")
    return {"reserved": reserved.value, "used": used.value}
