"""Input builder for tests and benchmarks: the reference's FDTD setup, restated.

Test and benchmark infrastructure, not part of the engine package. The
reference's own Python package (rfnetwork/solver.py, class ``FDTD_Solver``)
cannot be imported on this machine (pyvista, np_struct, skimage and
matplotlib are absent), so this module restates its setup code -- grid,
materials, PML grading, lumped ports, sources, probes, monitors and the
packing of ``solve()`` -- to produce, bit for bit, the coefficient arrays and
probe/monitor lists the reference's ``solve()`` hands its engine (pinned by
the fixtures under tests/golden/). The expressions and their order follow the
reference so that the float32 arrays are bit-equal; that is the reason for
the likeness. ``solve()`` runs the packed inputs through the engine's drop-in
``rfnetwork_b200.cuda_func``, as the reference's ``solve()`` does once the
shim is installed.

What is not carried over: the pyvista mesher (``generate_mesh`` takes the grid
edges, or a uniform cell width that divides the solve box exactly), gerber
image layers, rendering and the far-field transform. Geometry objects are the
axis-aligned primitives of ``modelgen.geometry``.
"""
from __future__ import annotations

import itertools
from copy import copy

import numpy as np

from rfnetwork_b200.units import const, conv

from . import geometry as geo

u0 = const.u0
e0 = const.e0
c0 = const.c0

FIELDS = ("ex", "ey", "ez", "hx", "hy", "hz")


def dtft(xn: np.ndarray, frequency: np.ndarray, fs: float, downsample: bool = False) -> np.ndarray:
    """Direct DTFT ``X(f) = sum_n x[n] exp(-j 2 pi f n / fs)`` (rfnetwork/utils.py:14-71).

    With ``downsample`` the series is low-passed (20th-order Butterworth,
    zero-phase) and decimated first, as the reference allows.
    """
    xn = np.asarray(xn)
    frequency = np.asarray(frequency)
    frs = np.max(frequency) * 20
    factor = int(fs / frs)
    use_ds = downsample and factor > 0 and (len(xn) / factor) > 100 and fs > (frs * 2)
    if use_ds:
        from scipy import signal

        sos = signal.butter(20, frs / 2.5, btype="lowpass", output="sos", fs=fs)
        xn = signal.sosfiltfilt(sos, xn)[::factor]
        fs = frs
    omega = 2 * np.pi * (frequency / fs)
    n = np.arange(len(xn))
    w_mesh, n_mesh = np.meshgrid(omega, n)
    Xw = np.sum(xn[..., None] * np.exp(-1j * w_mesh * n_mesh), axis=0)
    if use_ds:
        Xw *= factor
    return Xw


def _shift(a: np.ndarray, axis: int, lo: int) -> np.ndarray:
    """a without its first (lo=1) or last (lo=0) entry along ``axis``."""
    idx = [slice(None)] * a.ndim
    idx[axis] = slice(1, None) if lo else slice(None, -1)
    return a[tuple(idx)]


class FDTD_Solver:
    """FDTD EM solver for PCB geometries (reference: rfnetwork/solver.py:21)."""

    def __init__(self, bounding_box, courant: float = 0.95):
        """
        Parameters
        ----------
        bounding_box : geometry.Box
            box enclosing the solution space, inches.
        courant : float, default 0.95
            fraction of the 3D Courant limit used for the time step. The
            reference hard-codes 0.95 (rfnetwork/solver.py:883).
        """
        self.bounding_box = bounding_box
        self.dielectrics = dict()
        self.conductors = dict()
        self.lumped_elements = dict()
        self.pml_boundaries = []
        self.monitors = dict()
        self.farfield = dict()
        self.probes = dict()
        self.ports = []
        self.ports_inv = []
        self._n_pml = None
        self._auto_name_counter = 0
        self.sbox_max = np.max(bounding_box.points, axis=0)
        self.sbox_min = np.min(bounding_box.points, axis=0)
        self._places = 5
        self._tol = 1 / (10 ** self._places)
        self._courant = courant
        self._meshed = False
        self._solved = False
        self._time = None
        self.last_run = None

    # ------------------------------------------------------------------ state
    @property
    def time(self):
        return self._time

    def invalidate_mesh(self):
        self._meshed = False
        self.invalidate_solution()

    def invalidate_solution(self):
        self._solved = False

    def check_mesh(self):
        if not self._meshed:
            raise RuntimeError("Mesh has been invalidated or has not been created yet.")

    def check_solution(self):
        if not self._solved:
            raise RuntimeError("Solution has been invalidated or model has not been solved yet.")

    # ---------------------------------------------------------------- objects
    def _add_object(self, group, objects, properties, name=None):
        self.invalidate_mesh()
        if not isinstance(objects, (tuple, list, np.ndarray)):
            objects = [objects]
        if name is not None and name in self.conductors.keys():
            raise ValueError(f"Duplicate conductor name: {name}")
        for i, obj in enumerate(objects):
            if name is None:
                obj_name = f"obj_{self._auto_name_counter}"
                self._auto_name_counter += 1
            else:
                obj_name = name + "_{i}" if len(objects) > 1 else name
            group[obj_name] = dict(obj=obj, **properties)

    def add_dielectric(self, *objects, er: float, loss_tan: float = 0, f0: float = 0, style: dict = None,
                       name: str = None):
        """Add rectangular dielectric boxes (rfnetwork/solver.py:100-130)."""
        self._add_object(self.dielectrics, objects, dict(er=er, loss_tan=loss_tan, f0=f0), name=name)

    def add_conductor(self, *objects, sigma: float = 1e16, style: dict = None, name: str = None):
        """Add conductor boxes or sheets (rfnetwork/solver.py:132-148)."""
        self._add_object(self.conductors, objects, dict(sigma=sigma), name=name)

    def add_lumped_port(self, number: int, face, integration_line: str, r0: float = 50, name: str = None):
        """Attach a lumped port to a face (rfnetwork/solver.py:150-261), axis-notation form."""
        if not isinstance(integration_line, str):
            raise NotImplementedError("Only axis notation ('x+', 'z-', ...) integration lines are supported.")
        self._add_object(self.lumped_elements, face,
                         dict(integration_line=integration_line, r=r0, port=number), name=name)

    def add_resistor(self, face, value: float, integration_line: str, name: str = None):
        """Attach a resistive element to a face (rfnetwork/solver.py:263-282)."""
        self._add_object(self.lumped_elements, face,
                         dict(integration_line=integration_line, r=value, port=None), name=name)

    def assign_PML_boundaries(self, *sides: str, n_pml: int = 10):
        """Assign PML layers to sides of the solve box (rfnetwork/solver.py:362-382)."""
        self.invalidate_mesh()
        valid = ("x+", "x-", "y+", "y-", "z+", "z-")
        if any(s not in valid for s in sides):
            raise ValueError(f"PML side not recognized. Expecting one of {valid}")
        self.pml_boundaries = copy(list(sides))
        self._n_pml = n_pml

    # ------------------------------------------------------------- indexing
    def pos_to_idx(self, position, mode="edge"):
        """Index of the grid edge / cell centre on or just past ``position`` (solver.py:384-402)."""
        self.check_mesh()
        idx = []
        mode = [mode] * 3 if isinstance(mode, str) else mode
        grid = [self.g_edges[i] if m == "edge" else self.g_cells[i] for i, m in enumerate(mode)]
        for i, g in enumerate(grid):
            diff = g - position[i]
            idx += [np.argmax(diff >= -self._tol) if diff[-1] > -self._tol else len(g)]
        return tuple(idx)

    def edge_correction(self, p1, p2, integration_line: str, CFe: float = None, CFh: float = 1):
        """Analytic correction of the H updates next to a PEC edge (rfnetwork/solver.py:2534-2700).

        The fields near a thin conductor edge vary like 1/sqrt(distance), which
        the Yee cell integrals miss. Along the edge p1-p2 (parallel to one
        axis; ``integration_line`` the in-plane direction pointing away from the
        conductor) the H integration coefficients Db of the affected cells are
        scaled by CFe (default sqrt(2)) or 1/CFe, in the reference's order, so
        the packed coefficients match it bit for bit. CFh is accepted and, as in
        the reference, unused.
        """
        self.invalidate_solution()
        self.check_mesh()
        cf = 2 * np.sqrt(1 / 2) if CFe is None else CFe
        p1, p2 = np.array(p1), np.array(p2)
        length = np.abs(p2 - p1)
        if np.count_nonzero(length) != 1:
            raise NotImplementedError("Edge correction is only supported for edges along the cartesian axis.")
        ax_e = int(np.argmax(length))
        ax_f = dict(x=0, y=1, z=2)[integration_line[0]]
        outward = {"+": 1, "-": 0}[integration_line[1]]
        if ax_e == ax_f:
            raise ValueError("Integration axis must be perpendicular to the edge.")
        if p1[ax_e] > p2[ax_e]:
            p1, p2 = p2, p1
        i1, i2 = self.pos_to_idx(p1, mode="edge"), self.pos_to_idx(p2, mode="edge")
        ax_n = 3 - ax_e - ax_f
        e, f, nrm = ("x", "y", "z")[ax_e], ("x", "y", "z")[ax_f], ("x", "y", "z")[ax_n]
        Db = self.Db

        def at(along_edge, along_field, along_normal):
            sl = [None, None, None]
            sl[ax_e], sl[ax_f], sl[ax_n] = along_edge, along_field, along_normal
            return tuple(sl)

        centres = slice(i1[ax_e], i2[ax_e])      # components centred between edge nodes
        nodes = slice(i1[ax_e], i2[ax_e] + 1)    # components on the edge nodes
        h_f = i1[ax_f] if outward else i1[ax_f] - 1
        k_n = i1[ax_n]
        # the normal H in the conductor plane that integrates the field-axis E:
        # scaled down over the edge, up at the two ends
        Db[f"h{nrm}_{f}2"][at(centres, h_f, k_n)] *= 1 / cf
        Db[f"h{nrm}_{f}1"][at(centres, h_f, k_n)] *= 1 / cf
        if i1[ax_e] > 0:
            Db[f"h{nrm}_{e}2"][at(i1[ax_e] - 1, h_f, k_n)] *= cf
        if i2[ax_e] < Db[f"h{nrm}_{e}1"].shape[ax_e]:
            Db[f"h{nrm}_{e}1"][at(i2[ax_e], h_f, k_n)] *= cf
        # the edge-parallel H just below and above the conductor plane
        Db[f"h{e}_{nrm}2"][at(nodes, h_f, k_n - 1)] *= cf
        Db[f"h{e}_{nrm}1"][at(nodes, h_f, k_n)] *= cf
        for k in (k_n - 1, k_n):
            # edge-parallel H on both sides of the normal E under the edge
            Db[f"h{e}_{f}2"][at(nodes, i1[ax_f] - 1, k)] *= cf
            Db[f"h{e}_{f}1"][at(nodes, i1[ax_f], k)] *= cf
            # field-axis H that integrates the normal E below and above the edge
            Db[f"h{f}_{nrm}1"][at(centres, i1[ax_f], k)] *= 1 / cf
            Db[f"h{f}_{nrm}2"][at(centres, i1[ax_f], k)] *= 1 / cf
            if i1[ax_e] > 0:
                Db[f"h{f}_{e}2"][at(i1[ax_e] - 1, i1[ax_f], k)] *= cf
            if i2[ax_e] < Db[f"h{f}_{e}1"].shape[ax_e]:
                Db[f"h{f}_{e}1"][at(i2[ax_e], i1[ax_f], k)] *= cf

    def field_pos_to_idx(self, position, field):
        """Index of the ``field`` component on or just past ``position`` (solver.py:404-420)."""
        self.check_mesh()
        idx = []
        for i, g in enumerate(self.floc[field]):
            diff = g - position[i]
            idx += [np.argmax(diff >= -self._tol) if diff[-1] > -self._tol else len(g)]
        return tuple(idx)

    # ----------------------------------------------------------------- mesh
    def generate_mesh(self, d_max: float = None, d_min: float = None, grid=None):
        """Build the grid and all update coefficients (rfnetwork/solver.py:423-451).

        ``grid`` gives the cell edges (gx, gy, gz) in inches. Without it the
        solve box is cut into uniform cells of width ``d_max``, which must
        divide every side of the box.
        """
        if grid is None:
            if d_max is None:
                raise ValueError("generate_mesh needs d_max or explicit grid edges")
            grid = []
            for a in range(3):
                n = (float(self.sbox_max[a]) - float(self.sbox_min[a])) / d_max
                if abs(n - round(n)) > 1e-6:
                    raise ValueError("d_max must divide the solve box into whole cells")
                grid.append(float(self.sbox_min[a]) + d_max * np.arange(int(round(n)) + 1))
        self._meshed = True
        self._init_grid(grid)
        self._init_dielectrics()
        self._init_coefficients()
        for side in self.pml_boundaries:
            self._init_PML(side)
        self._init_conductors()
        self._init_lumped_elements()
        self.invalidate_solution()

    def _init_grid(self, grid):
        """Grid arrays (rfnetwork/solver.py:640-707, after the mesher has produced the edges)."""
        dtype_ = np.float32
        gx, gy, gz = [np.asarray(g, dtype=np.float64).astype(dtype_) for g in grid]
        self.g_edges_raw = (gx, gy, gz)
        dx, dy, dz = np.diff(gx).astype(dtype_), np.diff(gy).astype(dtype_), np.diff(gz).astype(dtype_)
        self.n_cells = len(dx), len(dy), len(dz)
        self.Nx, self.Ny, self.Nz = self.n_cells
        self.dx, self.dy, self.dz = dx, dy, dz
        gx_h, gy_h, gz_h = (gx[1:] + gx[:-1]) / 2, (gy[1:] + gy[:-1]) / 2, (gz[1:] + gz[:-1]) / 2
        dx_h, dy_h, dz_h = (dx[1:] + dx[:-1]) / 2, (dy[1:] + dy[:-1]) / 2, (dz[1:] + dz[:-1]) / 2
        self.g_edges = gx, gy, gz
        self.g_cells = gx_h, gy_h, gz_h
        self.d_cells = dx, dy, dz
        self.dh_cells = dx_h, dy_h, dz_h
        self.dx_h, self.dy_h, self.dz_h = dx_h, dy_h, dz_h
        self.eps = np.ones(self.n_cells) * e0
        self.sigma = np.zeros(self.n_cells)
        self.floc = dict(ex=(gx_h, gy, gz), ey=(gx, gy_h, gz), ez=(gx, gy, gz_h),
                         hx=(gx, gy_h, gz_h), hy=(gx_h, gy, gz_h), hz=(gx_h, gy_h, gz))
        Nx, Ny, Nz = self.n_cells
        self.fshape = dict(ex=(Nx, Ny + 1, Nz + 1), ey=(Nx + 1, Ny, Nz + 1), ez=(Nx + 1, Ny + 1, Nz),
                           hx=(Nx + 1, Ny, Nz), hy=(Nx, Ny + 1, Nz), hz=(Nx, Ny, Nz + 1))
        dx_hp, dy_hp, dz_hp = np.pad(dx_h, (1, 1)), np.pad(dy_h, (1, 1)), np.pad(dz_h, (1, 1))
        self.fcell_w = dict(ex=(dx, dy_hp, dz_hp), ey=(dx_hp, dy, dz_hp), ez=(dx_hp, dy_hp, dz),
                            hx=(dx_hp, dy, dz), hy=(dx, dy_hp, dz), hz=(dx, dy, dz_hp))

    def _init_dielectrics(self):
        """Per-cell permittivity / conductivity, max rule on overlap (solver.py:794-815)."""
        for sub in self.dielectrics.values():
            if sub["obj"].n_cells > 6:
                raise NotImplementedError("Only rectangular dielectrics are supported.")
            x0, y0, z0 = self.pos_to_idx(np.min(sub["obj"].points, axis=0), mode="cell")
            x1, y1, z1 = self.pos_to_idx(np.max(sub["obj"].points, axis=0), mode="cell")
            region = (slice(x0, x1), slice(y0, y1), slice(z0, z1))
            cur = self.eps[region]
            self.eps[region] = np.where(cur > e0 * sub["er"], cur, e0 * sub["er"])
            sub_sigma = sub["loss_tan"] * e0 * sub["er"] * 2 * np.pi * sub["f0"]
            cur = self.sigma[region]
            self.sigma[region] = np.where(cur > sub_sigma, cur, sub_sigma)

    def _init_coefficients(self):
        """Time step and base E/H coefficients (rfnetwork/solver.py:871-1003)."""
        dtype_ = np.float32
        dx, dy, dz = [conv.m_in(d) for d in self.d_cells]
        Nx, Ny, Nz = self.n_cells
        length_min = np.array([np.min(dx), np.min(dy), np.min(dz)], dtype=dtype_)
        dmin = 1 / np.sqrt(((1 / length_min) ** 2).sum())
        dt = self._courant * (dmin / const.c0)
        self.dt = dt
        Cb_0 = dt / e0
        Db_0 = dt / u0

        def edge_average(v):
            # average adjacent cells onto the cell edges / faces, weighted by half widths
            dx0, dx1 = dx[:-1][..., None, None], dx[1:][..., None, None]
            dy0, dy1 = dy[:-1][None, :, None], dy[1:][None, :, None]
            dz0, dz1 = dz[:-1][None, None], dz[1:][None, None]
            v_x = (v[:-1] * (dx0 / 2) + v[1:] * (dx1 / 2)) / (dx0 / 2 + dx1 / 2)
            v_y = (v[:, :-1] * (dy0 / 2) + v[:, 1:] * (dy1 / 2)) / (dy0 / 2 + dy1 / 2)
            v_z = (v[..., :-1] * (dz0 / 2) + v[..., 1:] * (dz1 / 2)) / (dz0 / 2 + dz1 / 2)
            v_yz = (v_y[..., :-1] * (dz0 / 2) + v_y[..., 1:] * (dz1 / 2)) / (dz0 / 2 + dz1 / 2)
            v_xz = (v_x[..., :-1] * (dz0 / 2) + v_x[..., 1:] * (dz1 / 2)) / (dz0 / 2 + dz1 / 2)
            v_xy = (v_x[:, :-1] * (dy0 / 2) + v_x[:, 1:] * (dy1 / 2)) / (dy0 / 2 + dy1 / 2)
            return v_x, v_y, v_z, v_xy, v_xz, v_yz

        eps_x, eps_y, eps_z, eps_xy, eps_xz, eps_yz = edge_average(self.eps)
        sig_x, sig_y, sig_z, sig_xy, sig_xz, sig_yz = edge_average(self.sigma)
        fs = self.fshape
        self.eps_ex = np.ones(fs["ex"], dtype=dtype_) * e0
        self.eps_ey = np.ones(fs["ey"], dtype=dtype_) * e0
        self.eps_ez = np.ones(fs["ez"], dtype=dtype_) * e0
        self.eps_ex[:, 1:-1, 1:-1] = eps_yz
        self.eps_ey[1:-1, :, 1:-1] = eps_xz
        self.eps_ez[1:-1, 1:-1] = eps_xy
        self.eps_hx = np.ones(fs["hx"], dtype=dtype_) * e0
        self.eps_hy = np.ones(fs["hy"], dtype=dtype_) * e0
        self.eps_hz = np.ones(fs["hz"], dtype=dtype_) * e0
        self.eps_hx[1:-1, ] = eps_x
        self.eps_hy[:, 1:-1] = eps_y
        self.eps_hz[..., 1:-1] = eps_z
        self.sig_ex = np.zeros(fs["ex"], dtype=dtype_)
        self.sig_ey = np.zeros(fs["ey"], dtype=dtype_)
        self.sig_ez = np.zeros(fs["ez"], dtype=dtype_)
        self.sig_ex[:, 1:-1, 1:-1] = sig_yz
        self.sig_ey[1:-1, :, 1:-1] = sig_xz
        self.sig_ez[1:-1, 1:-1] = sig_xy

        def ca(eps, sig):
            return (2 * eps - (sig * dt)) / (2 * eps + (sig * dt))

        def cb(eps, sig):
            return (2 * dt) / ((2 * eps + (sig * dt)))

        Ca_ex, Ca_ey, Ca_ez = ca(self.eps_ex, self.sig_ex), ca(self.eps_ey, self.sig_ey), ca(self.eps_ez, self.sig_ez)
        Cb_ex, Cb_ey, Cb_ez = cb(self.eps_ex, self.sig_ex), cb(self.eps_ey, self.sig_ey), cb(self.eps_ez, self.sig_ez)
        self.Ca = dict(ex_y=Ca_ex.copy(), ex_z=Ca_ex.copy(), ey_z=Ca_ey.copy(), ey_x=Ca_ey.copy(),
                       ez_x=Ca_ez.copy(), ez_y=Ca_ez.copy())
        self.Cb = dict(ex_y=Cb_ex.copy(), ex_z=Cb_ex.copy(), ey_z=Cb_ey.copy(), ey_x=Cb_ey.copy(),
                       ez_x=Cb_ez.copy(), ez_y=Cb_ez.copy())
        hs = dict(hx=(Nx + 1, Ny, Nz), hy=(Nx, Ny + 1, Nz), hz=(Nx, Ny, Nz + 1))
        splits = dict(hx=("y", "z"), hy=("z", "x"), hz=("x", "y"))
        self.Da, self.Db = {}, {}
        for h, (a, b) in splits.items():
            for s in (a, b):
                self.Da[f"{h}_{s}"] = np.ones(hs[h], dtype=dtype_) * 1
                self.Db[f"{h}_{s}1"] = np.ones(hs[h], dtype=dtype_) * Db_0
                self.Db[f"{h}_{s}2"] = np.ones(hs[h], dtype=dtype_) * Db_0
        self._Cb_0 = Cb_0

    def _init_PML(self, side: str):
        """Graded split-field PML on one side (rfnetwork/solver.py:1239-1326)."""
        n_pml = self._n_pml
        if n_pml is None:
            return
        axis = side[0]
        axis_i = dict(x=0, y=1, z=2)[axis]
        m_pml = 3
        dt = self.dt
        dcells = self.d_cells[axis_i]
        d_border = conv.m_in(dcells[-1]) if side[1] == "+" else conv.m_in(dcells[0])
        eta0 = np.sqrt(u0 / e0)
        sigma_max = 0.8 * (m_pml + 1) / (eta0 * d_border)
        bshape = [None] * 3
        bshape[axis_i] = slice(None)
        i_pml = np.arange(0, n_pml)[tuple(bshape)]
        sigma_e_n = sigma_max * ((i_pml) / (n_pml)) ** m_pml
        sigma_e_np5 = sigma_max * ((i_pml + 0.5) / (n_pml)) ** m_pml
        e_idx = [slice(None)] * 3
        h_idx = [slice(None)] * 3
        e_idx[axis_i] = slice(n_pml, 0, -1) if side[1] == "-" else slice(-n_pml - 1, -1)
        h_idx[axis_i] = slice(n_pml - 1, None, -1) if side[1] == "-" else slice(-n_pml, None)
        e_idx, h_idx = tuple(e_idx), tuple(h_idx)
        field_eps = dict(ex=self.eps_ex, ey=self.eps_ey, ez=self.eps_ez,
                         hx=self.eps_hx, hy=self.eps_hy, hz=self.eps_hz)
        pml_efields = [("ey", "ez"), ("ez", "ex"), ("ex", "ey")][axis_i]
        pml_hfields = [("hy", "hz"), ("hz", "hx"), ("hx", "hy")][axis_i]
        for e in pml_efields:
            eps = field_eps[e][e_idx]
            sigma_e = np.broadcast_to(sigma_e_n, eps.shape).copy()
            sigma_e *= (eps / e0)
            self.Ca[f"{e}_{axis}"][e_idx] = (2 * eps - (sigma_e * dt)) / (2 * eps + (sigma_e * dt))
            self.Cb[f"{e}_{axis}"][e_idx] = (2 * dt) / ((2 * eps + (sigma_e * dt)))
        for h in pml_hfields:
            eps = field_eps[h][h_idx]
            sigma_e = np.broadcast_to(sigma_e_np5, eps.shape).copy()
            sigma_e *= (eps / e0)
            sigma_m = sigma_e * u0 / eps
            self.Da[f"{h}_{axis}"][h_idx] = (2 * u0 - (sigma_m * dt)) / (2 * u0 + (sigma_m * dt))
            self.Db[f"{h}_{axis}1"][h_idx] = (2 * dt) / ((2 * u0 + (sigma_m * dt)))
            self.Db[f"{h}_{axis}2"][h_idx] = (2 * dt) / ((2 * u0 + (sigma_m * dt)))

    def _init_conductors(self):
        """Conductor E coefficients, overriding the PML (rfnetwork/solver.py:817-869)."""
        e_eps = dict(ex=self.eps_ex, ey=self.eps_ey, ez=self.eps_ez)
        e_split = dict(ex=("ex_y", "ex_z"), ey=("ey_z", "ey_x"), ez=("ez_x", "ez_y"))
        for cond in self.conductors.values():
            obj, sig = cond["obj"], cond["sigma"]
            for field in ("ex", "ey", "ez"):
                p0 = list(self.field_pos_to_idx(np.min(obj.points, axis=0), field))
                p1 = list(self.field_pos_to_idx(np.max(obj.points, axis=0), field))
                bbox_idx = tuple(slice(p0[i], p1[i] + 1) for i in range(3))
                pts = np.meshgrid(*[self.floc[field][i][bbox_idx[i]] for i in range(3)], indexing="ij")
                pts = np.stack(pts, axis=-1)
                if geo.is_object_surface(obj):
                    inside = geo.points_in_rectangle(pts, obj, self._tol)
                else:
                    inside = (obj.implicit_distance(pts) - self._tol) <= 0
                eps_bbox = e_eps[field][bbox_idx]
                Ca_c = (2 * eps_bbox - (sig * self.dt)) / (2 * eps_bbox + (sig * self.dt))
                Cb_c = (2 * self.dt) / ((2 * eps_bbox + (sig * self.dt)))
                for e_sp in e_split[field]:
                    self.Ca[e_sp][bbox_idx] = np.where(inside, Ca_c, self.Ca[e_sp][bbox_idx])
                    self.Cb[e_sp][bbox_idx] = np.where(inside, Cb_c, self.Cb[e_sp][bbox_idx])

    def _init_lumped_elements(self):
        """Resistive sheets and lumped ports (rfnetwork/solver.py:1086-1237)."""
        ports = [el for el in self.lumped_elements.values() if el["port"] is not None]
        if not len(ports):
            return
        n_ports = max(abs(el["port"]) for el in ports)
        self.ports = [None] * n_ports
        self.ports_inv = [None] * n_ports
        d_cells = [conv.m_in(d) for d in self.d_cells]
        dh_cells = [conv.m_in(d) for d in self.dh_cells]
        for name, element in self.lumped_elements.items():
            face = element["obj"]
            r = element["r"]
            integration_line = element["integration_line"]
            port = element["port"]
            if face.n_cells > 1 or face.faces[0] != 4:
                raise ValueError("Only rectangular port faces are supported.")
            p1 = np.array(self.pos_to_idx(np.min(face.points, axis=0), mode="edge"))
            p2 = np.array(self.pos_to_idx(np.max(face.points, axis=0), mode="edge"))
            idx_d = p2 - p1
            n_axis = np.argmin(idx_d)
            if np.count_nonzero(idx_d) != 2:
                raise ValueError("Port face must be on cartesian grid, and must be 2D.")
            f_axis = dict(x=0, y=1, z=2)[integration_line[0]]
            f_dir = {"+": 1, "-": -1}[integration_line[1]]
            w_axis = [ax for ax in (0, 1, 2) if ax != f_axis and ax != n_axis][0]
            if port is not None and idx_d[w_axis] < 2:
                raise NotImplementedError("Port faces must span at least 2 grid cells.")
            if port is not None:
                p1[w_axis] += 1
                p2[w_axis] -= 1
            if f_axis == n_axis:
                raise ValueError("Integration direction must be in the port face.")
            na, wa, fa = [["x", "y", "z"][ax] for ax in (n_axis, w_axis, f_axis)]

            def build_idx(normal, width, field):
                idx = [slice(None)] * 3
                idx[w_axis] = width
                idx[f_axis] = field
                idx[n_axis] = normal
                return tuple(idx)

            dw = dh_cells[w_axis][p1[w_axis] - 1: p2[w_axis]]
            dn = dh_cells[n_axis][p1[n_axis] - 1: p2[n_axis]]
            df = d_cells[f_axis][p1[f_axis]: p2[f_axis]]
            gx_, gy_, gz_ = np.meshgrid(*build_idx(dn, dw, df), indexing="ij")
            dn, dw, df = [(gx_, gy_, gz_)[ax] for ax in (n_axis, w_axis, f_axis)]
            eps_field = [self.eps_ex, self.eps_ey, self.eps_ez][f_axis]
            efield_idx = build_idx(slice(p1[n_axis], p2[n_axis] + 1), slice(p1[w_axis], p2[w_axis] + 1),
                                   slice(p1[f_axis], p2[f_axis]))
            eps_r = eps_field[efield_idx]
            nw = (p2 - p1 + 1)[w_axis]
            nf = (p2 - p1)[f_axis]
            r_cell = r * (nw) / nf
            rterm = (r_cell * dn * dw)
            denom = (eps_r / self.dt) + (df / (2 * rterm))
            self.Ca[f"e{fa}_{wa}"][efield_idx] = ((eps_r / self.dt) - (df / (2 * rterm))) / denom
            self.Cb[f"e{fa}_{wa}"][efield_idx] = 1 / (denom)
            self.Ca[f"e{fa}_{na}"][efield_idx] = ((eps_r / self.dt) - (df / (2 * rterm))) / denom
            self.Cb[f"e{fa}_{na}"][efield_idx] = 1 / (denom)
            if port is not None:
                group = self.ports if port > 0 else self.ports_inv
                group[abs(port) - 1] = dict(idx=efield_idx, Vs_a=-f_dir / (denom * rterm * nf), field=f"e{fa}",
                                            axis=n_axis, r0=r, direction=f_dir, src=None)
                fpos1 = np.min(face.points, axis=0)
                fpos2 = np.max(face.points, axis=0)
                field_loc = self.floc[f"e{fa}"][f_axis]
                fpos_n = field_loc[int((p2 + p1)[f_axis] / 2)]
                current_face = geo.Rectangle([
                    build_idx(fpos1[n_axis] - 0.001, fpos1[w_axis] - 0.001, fpos_n),
                    build_idx(fpos1[n_axis] - 0.001, fpos2[w_axis] + 0.001, fpos_n),
                    build_idx(fpos1[n_axis] + 0.001, fpos2[w_axis] + 0.001, fpos_n),
                ])
                self.add_current_probe(f"port_{port}", current_face)

    # -------------------------------------------------------------- sources
    def gaussian_source(self, width: float, t0: float, t_len: float) -> np.ndarray:
        """Unit-amplitude Gaussian pulse (rfnetwork/solver.py:1328-1342)."""
        n_len = int(t_len / self.dt)
        t = np.linspace(0, self.dt * n_len, n_len)
        vsrc = np.exp(-((t - t0) / (width / 4)) ** 2)
        return vsrc / np.max(np.abs(vsrc))

    def gaussian_modulated_source(self, f0: float, width: float, t0: float, t_len: float) -> np.ndarray:
        """Unit-amplitude Gaussian-modulated sinusoid (rfnetwork/solver.py:1344-1358)."""
        n_len = int(t_len / self.dt)
        t = np.linspace(0, self.dt * n_len, n_len)
        vsrc = np.exp(-((t - t0) / (width / 4)) ** 2) * np.sin(2 * np.pi * f0 * t)
        return vsrc / np.max(np.abs(vsrc))

    def assign_excitation(self, waveform: np.ndarray, ports):
        """Assign a voltage waveform to ports (rfnetwork/solver.py:1360-1396)."""
        self.invalidate_solution()
        self.check_mesh()
        if self._time is None:
            self._time = np.arange(0, self.dt * len(waveform), self.dt)
        if len(self._time) > len(waveform):
            pad = np.zeros_like(self._time)
            pad[:len(waveform)] = waveform
            waveform = pad
        if len(self._time) < len(waveform):
            waveform = waveform[:len(self._time)]
        for p in np.atleast_1d(ports):
            self.ports[p - 1]["src"] = waveform.astype(np.float32)
            if self.ports_inv[p - 1] is not None:
                self.ports_inv[p - 1]["src"] = waveform.astype(np.float32)

    def reset_excitations(self):
        self._time = None
        for p in self.ports:
            p["src"] = None
        for p in self.ports_inv:
            if p is not None:
                p["src"] = None

    # ---------------------------------------------------------- probes / mon
    def add_field_monitor(self, name: str, field: str, axis: str, position: float = None, index: int = None,
                          n_step: int = 1, frequency=None):
        """Plane field monitor, time samples or phasors (rfnetwork/solver.py:1703-1775)."""
        supported = tuple(self.fshape.keys()) + ("e_total",)
        if field not in supported:
            raise ValueError(f"Unsupported field: {field}. Expecting one of: {supported}")
        if axis not in ("x", "y", "z"):
            raise ValueError(f"Unsupported axis: {axis}")
        axis_i = dict(x=0, y=1, z=2)[axis]
        if field == "e_total":
            fields, names = ("ex", "ey", "ez"), [name + "_" + f for f in ("x", "y", "z")]
        else:
            fields, names = [field], [name]
        for n, f in zip(names, fields):
            shape = list(self.fshape[f])
            axis_len = shape.pop(axis_i)
            idx = index
            pos = position
            if pos is not None:
                full = [0] * 3
                full[axis_i] = pos
                idx = int(self.field_pos_to_idx(full, f)[axis_i])
            elif idx is not None:
                pos = self.floc[f][axis_i][idx]
            if idx < 0 or idx >= (axis_len - 1):
                raise ValueError("Field position out of bounds")
            self.monitors[n] = dict(field=f, axis=axis_i, position=pos, index=idx, n_step=n_step,
                                    shape=tuple(shape),
                                    frequency=np.atleast_1d(frequency) if frequency is not None else None)

    def add_farfield_monitor(self, frequency, padding: int = 2):
        """Phasor monitors on the faces of a box ``padding`` cells inside the PML
        (rfnetwork/solver.py:1777-1891): per face with PML, the two tangential E
        components on the face plane and the two tangential H components on the
        planes either side of it (averaged onto the face later). Faces on a side
        without PML sit on the grid boundary and get no monitors."""
        self.check_mesh()
        if not len(self.pml_boundaries):
            raise ValueError("No radiation or PML boundaries found. Unable to create farfield monitor.")
        ff_idx = np.zeros((3, 2), dtype=np.int64)
        surf_pos = np.zeros((3, 2), dtype=np.float64)
        for axis in range(3):
            a = "xyz"[axis]
            tangential = [i for i in (0, 1, 2) if i != axis]
            for j, side in enumerate(("n", "p")):
                n_edges = len(self.g_edges[axis])
                has_pml = (a + ("-" if side == "n" else "+")) in self.pml_boundaries
                if has_pml:
                    ff_idx[axis, j] = self._n_pml + padding if j == 0 else n_edges - self._n_pml - 1 - padding
                else:
                    ff_idx[axis, j] = 0 if j == 0 else n_edges - 1
                k = int(ff_idx[axis, j])
                surf_pos[axis, j] = conv.m_in(self.g_edges[axis][k])
                if not has_pml:
                    continue
                for f in tangential:
                    fs = "xyz"[f]
                    self.add_field_monitor(f"ff_e{fs}_{side}{a}", f"e{fs}", a, index=k, frequency=frequency)
                    self.add_field_monitor(f"ff_h{fs}1_{side}{a}", f"h{fs}", a, index=k, frequency=frequency)
                    self.add_field_monitor(f"ff_h{fs}2_{side}{a}", f"h{fs}", a, index=k - 1 if j == 0 else k + 1,
                                           frequency=frequency)
        cell_pos, cell_w = [None] * 3, [None] * 3
        for axis in range(3):
            f0, f1 = [i for i in (0, 1, 2) if i != axis]
            s0 = slice(int(ff_idx[f0, 0]), int(ff_idx[f0, 1]))
            s1 = slice(int(ff_idx[f1, 0]), int(ff_idx[f1, 1]))
            cell_pos[axis] = np.meshgrid(conv.m_in(self.g_cells[f0][s0]), conv.m_in(self.g_cells[f1][s1]),
                                         indexing="ij")
            cell_w[axis] = np.meshgrid(conv.m_in(self.d_cells[f0][s0]), conv.m_in(self.d_cells[f1][s1]),
                                       indexing="ij")
        self.farfield = dict(surf_pos=surf_pos, cell_pos=cell_pos, cell_w=cell_w, idx=ff_idx,
                             frequency=np.atleast_1d(frequency))

    def farfield_currents(self):
        """Equivalent surface currents of the far-field monitors at the face
        cell centers, in the argument layout of the far-field transform
        (rfnetwork/solver.py:2897-2999): J = n x H, M = -n x E, H averaged
        between its two planes and both fields averaged onto the cell centers."""
        self.check_solution()
        if not len(self.farfield):
            raise RuntimeError("Far-field monitor not found.")
        ff_idx = self.farfield["idx"]
        F = len(self.farfield["frequency"])
        J_xyz = [[None, None] for _ in range(3)]
        M_xyz = [[None, None] for _ in range(3)]
        surf_pos = [[None, None] for _ in range(3)]
        r_grid = [[None, None] for _ in range(3)]
        ds_grid = [None] * 3
        for axis in range(3):
            a = "xyz"[axis]
            f0, f1 = [i for i in (0, 1, 2) if i != axis]
            r_grid[axis][0] = np.array(self.farfield["cell_pos"][axis][0], dtype=np.float32, order="C")
            r_grid[axis][1] = np.array(self.farfield["cell_pos"][axis][1], dtype=np.float32, order="C")
            ds_grid[axis] = np.array(self.farfield["cell_w"][axis][0] * self.farfield["cell_w"][axis][1],
                                     dtype=np.complex64, order="C")
            shape = self.farfield["cell_pos"][axis][0].shape
            s0 = slice(int(ff_idx[f0, 0]), int(ff_idx[f0, 1]))
            s1 = slice(int(ff_idx[f1, 0]), int(ff_idx[f1, 1]))
            for j, side in enumerate(("n", "p")):
                surf_pos[axis][j] = self.farfield["surf_pos"][axis, j]
                e_xyz = np.zeros((3, F) + shape, dtype=np.complex64)
                h_xyz = np.zeros((3, F) + shape, dtype=np.complex64)
                for f in (f0, f1):
                    fs = "xyz"[f]
                    emon, hmon1, hmon2 = f"ff_e{fs}_{side}{a}", f"ff_h{fs}1_{side}{a}", f"ff_h{fs}2_{side}{a}"
                    if emon not in self.monitors:
                        continue
                    e = self.get_monitor_data(emon)[0]
                    h1, h2 = self.get_monitor_data(hmon1)[0], self.get_monitor_data(hmon2)[0]
                    w1 = self.d_cells[axis][self.monitors[hmon1]["index"]]
                    w2 = self.d_cells[axis][self.monitors[hmon2]["index"]]
                    h = (h1 * (w1 / 2) + h2 * (w2 / 2)) / ((w1 / 2) + (w2 / 2))
                    # E: average along the other tangential axis; H: along its own
                    e_ax = 1 if f == f1 else 2
                    h_ax = 1 if f == f0 else 2
                    e_c = (_shift(e, e_ax, 1) + _shift(e, e_ax, 0)) / 2
                    h_c = (_shift(h, h_ax, 1) + _shift(h, h_ax, 0)) / 2
                    e_xyz[f] = e_c[:, s0, s1]
                    h_xyz[f] = h_c[:, s0, s1]
                normal = np.array([0, 0, 0])
                normal[axis] = -1 if j == 0 else 1
                J_xyz[axis][j] = np.array(np.cross(normal, h_xyz, axis=0), order="C", dtype=np.complex64)
                M_xyz[axis][j] = np.array(np.cross(-normal, e_xyz, axis=0), order="C", dtype=np.complex64)
        return J_xyz, M_xyz, r_grid, ds_grid, surf_pos

    def get_farfield_rE(self, theta, phi) -> np.ndarray:
        """Far-field E (theta and phi polarisations) normalised by exp(-j beta r) / r,
        [2, frequency, theta, phi] complex64, theta and phi in degrees
        (rfnetwork/solver.py:2870-3021); the transform runs on the GPU engine."""
        from rfnetwork_b200 import _lib

        theta, phi = np.atleast_1d(theta), np.atleast_1d(phi)
        J_xyz, M_xyz, r_grid, ds_grid, surf_pos = self.farfield_currents()
        frequency = self.farfield["frequency"]
        ff_data = dict(
            beta=np.array(2 * np.pi * frequency / const.c0, dtype=np.float32),
            theta=np.array(np.deg2rad(theta), dtype=np.float32),
            phi=np.array(np.deg2rad(phi), dtype=np.float32),
            data=np.zeros((2, len(frequency), len(theta), len(phi)), dtype=np.complex64),
        )
        _lib.nf2ff(J_xyz, M_xyz, r_grid, ds_grid, surf_pos, ff_data)
        return ff_data["data"]

    def get_farfield_gain(self, theta, phi, polarization=None) -> np.ndarray:
        """Realized gain [polarization, frequency, theta, phi] from the far-field
        monitor (rfnetwork/solver.py:2804-2868): the far field projected on each
        polarization ("thetapol", "phipol", "rhcp", "lhcp"; default the first
        two), radiation intensity |rE|^2 / (2 eta0), over the power the port
        sources deliver into 50 ohm, |DTFT(v_src)|^2 / 100 summed over sources,
        times 4 pi."""
        rE = self.get_farfield_rE(theta, phi)
        if polarization is None:
            polarization = ["thetapol", "phipol"]
        s2 = 1 / np.sqrt(2)
        basis = dict(thetapol=[1, 0], phipol=[0, 1], rhcp=[s2, 1j * s2], lhcp=[s2, -1j * s2])
        proj = np.array([basis[k] for k in polarization])
        rE_pol = np.einsum("ij, j...->i...", proj, rE)
        frequency = self.farfield["frequency"]
        sources = [p["src"] for p in self.ports if p["src"] is not None]
        Vs = np.array([dtft(v, frequency, 1 / self.dt, downsample=False) for v in sources])
        p_in = np.sum((1 / 2) * (np.abs(Vs) ** 2 / 50), axis=0)
        U = (1 / (2 * const.eta0)) * np.abs(rE_pol) ** 2
        return (4 * np.pi / p_in[None, :, None, None]) * U

    def add_current_probe(self, name: str, face):
        """Ampere-loop H probes around a rectangle (rfnetwork/solver.py:1893-2010)."""
        dx_h, dy_h, dz_h = [conv.m_in(d) for d in self.dh_cells]
        if face.n_cells > 1 or face.faces[0] != 4:
            raise ValueError("Only rectangular current faces are supported.")
        pmin, pmax = np.min(face.points, axis=0), np.max(face.points, axis=0)
        face_size = pmax - pmin
        axis = np.argmin(face_size)
        if np.count_nonzero(face_size) != 2:
            raise ValueError("Port face must be on cartesian grid, and must be 2D.")
        # (axis, loop fields): for current along `axis`, the loop uses two H
        # components; "a" runs along the first in-plane axis, "b" the second.
        i = 0
        if axis == 0:
            x0 = self.field_pos_to_idx(pmin, "hy")[0]
            hz_y0 = self.field_pos_to_idx(pmin, "hz")[1] - 1
            hz_y1 = self.field_pos_to_idx(pmax, "hz")[1]
            hy_y = np.arange(hz_y0 + 1, hz_y1 + 1)
            hy_z0 = self.field_pos_to_idx(pmin, "hy")[2] - 1
            hy_z1 = self.field_pos_to_idx(pmax, "hy")[2]
            hz_z = np.arange(hy_z0 + 1, hy_z1 + 1)
            for z in hz_z:
                self.probes[f"{name}_{i}"] = dict(field="hz", index=(x0, hz_y0, z), d=-dz_h[z - 1]); i += 1
                self.probes[f"{name}_{i}"] = dict(field="hz", index=(x0, hz_y1, z), d=dz_h[z - 1]); i += 1
            for y in hy_y:
                self.probes[f"{name}_{i}"] = dict(field="hy", index=(x0, y, hy_z0), d=dy_h[y - 1]); i += 1
                self.probes[f"{name}_{i}"] = dict(field="hy", index=(x0, y, hy_z1), d=-dy_h[y - 1]); i += 1
        elif axis == 1:
            y0 = self.field_pos_to_idx(pmin, "hz")[1]
            hx_z0 = self.field_pos_to_idx(pmin, "hx")[2] - 1
            hx_z1 = self.field_pos_to_idx(pmax, "hx")[2]
            hz_z = np.arange(hx_z0 + 1, hx_z1 + 1)
            hz_x0 = self.field_pos_to_idx(pmin, "hz")[0] - 1
            hz_x1 = self.field_pos_to_idx(pmax, "hz")[0]
            hx_x = np.arange(hz_x0 + 1, hz_x1 + 1)
            for z in hz_z:
                self.probes[f"{name}_{i}"] = dict(field="hz", index=(hz_x0, y0, z), d=dz_h[z - 1]); i += 1
                self.probes[f"{name}_{i}"] = dict(field="hz", index=(hz_x1, y0, z), d=-dz_h[z - 1]); i += 1
            for x in hx_x:
                self.probes[f"{name}_{i}"] = dict(field="hx", index=(x, y0, hx_z0), d=-dx_h[x - 1]); i += 1
                self.probes[f"{name}_{i}"] = dict(field="hx", index=(x, y0, hx_z1), d=dx_h[x - 1]); i += 1
        elif axis == 2:
            z0 = self.field_pos_to_idx(pmin, "hx")[2]
            hx_y0 = self.field_pos_to_idx(pmin, "hx")[1] - 1
            hx_y1 = self.field_pos_to_idx(pmax, "hx")[1]
            hy_y = np.arange(hx_y0 + 1, hx_y1 + 1)
            hy_x0 = self.field_pos_to_idx(pmin, "hy")[0] - 1
            hy_x1 = self.field_pos_to_idx(pmax, "hy")[0]
            hx_x = np.arange(hy_x0 + 1, hy_x1 + 1)
            for y in hy_y:
                self.probes[f"{name}_{i}"] = dict(field="hy", index=(hy_x0, y, z0), d=-dy_h[y - 1]); i += 1
                self.probes[f"{name}_{i}"] = dict(field="hy", index=(hy_x1, y, z0), d=dy_h[y - 1]); i += 1
            for x in hx_x:
                self.probes[f"{name}_{i}"] = dict(field="hx", index=(x, hx_y0, z0), d=dx_h[x - 1]); i += 1
                self.probes[f"{name}_{i}"] = dict(field="hx", index=(x, hx_y1, z0), d=-dx_h[x - 1]); i += 1
        else:
            raise ValueError("Unrecognized axis.")

    def add_point_probe(self, name: str, field: str, index, d: float = 1.0):
        """Record one field component at a full-grid component index.

        Not in the reference API; it is the single-component case of
        ``add_voltage_probe`` / ``add_current_probe`` (one probe dict,
        rfnetwork/solver.py:2078-2080), used by the point-probe workloads.
        """
        if field not in FIELDS:
            raise ValueError(f"Unsupported field: {field}")
        self.probes[name] = dict(field=field, index=tuple(int(i) for i in index), d=d)

    def add_soft_source(self, name: str, field: str, index, waveform: np.ndarray):
        """Soft source on one field component: the waveform is added to both
        split fields each step, exactly as a port component's source probe is
        (solver.cpp:962-976). Not in the reference API, which only drives
        lumped ports; it serves point-source workloads."""
        if field not in FIELDS:
            raise ValueError(f"Unsupported field: {field}")
        self.soft_sources = getattr(self, "soft_sources", {})
        self.soft_sources[name] = dict(field=field, index=tuple(int(i) for i in index),
                                       src=np.asarray(waveform, dtype=np.float32))
        self.invalidate_solution()

    def add_voltage_probe(self, name: str, line):
        """E-field line probe for V = -int E dl (rfnetwork/solver.py:2012-2080)."""
        line_length = np.diff(line.points, axis=0)
        if np.count_nonzero(line_length) != 1:
            raise ValueError("Voltage probe must be parallel to the caresian axes.")
        axis = np.argmax(np.any(line_length, axis=0))
        field = ["ex", "ey", "ez"][axis]
        if len(line.points) != 2:
            raise ValueError("Voltage probe must be a line.")
        line_start, line_end = np.min(line.points, axis=0), np.max(line.points, axis=0)
        ijk_start = list(self.field_pos_to_idx(line_start, field))
        ijk_end = list(self.field_pos_to_idx(line_end, field))
        if self.floc[field][axis][ijk_end[axis]] > (line_end[axis] + self._tol):
            ijk_end[axis] -= 1
        n_probes = ijk_end[axis] - ijk_start[axis] + 1
        ijk = np.broadcast_to(ijk_start, (n_probes, 3)).copy()
        ijk[:, axis] = np.arange(ijk_start[axis], ijk_end[axis] + 1)
        fcell_w = self.fcell_w[field]
        p1, p2 = line.points
        direction = -1 if p1[axis] > p2[axis] else 1
        for i, idx in enumerate(ijk):
            cw = [fcell_w[a][j] for a, j in enumerate(idx)][axis]
            self.probes[f"{name}_{i}"] = dict(field=field, index=(idx), d=(direction) * conv.m_in(cw))

    # ---------------------------------------------------------------- solve
    def pack_inputs(self, gpu: bool = True, n_threads: int = 4):
        """Marshal the model into the engine arguments (rfnetwork/solver.py:1426-1622).

        Returns ``(coefficients, probes, monitors, mem, Nx, Ny, Nz, Nt)``:
        with ``gpu=True`` every coefficient array has shape (Nx, Ny, Nz) (the
        CUDA engine's form); with ``gpu=False`` the CPU engine's trimmed shapes.
        """
        self.check_mesh()
        soft = getattr(self, "soft_sources", {})
        excitations = [p["src"] for p in self.ports if p["src"] is not None]
        excitations += [v["src"] for v in soft.values()]
        if not len(excitations):
            raise ValueError("No port excitations found.")
        Nt = len(excitations[0])
        if not all(Nt == len(s) for s in excitations):
            raise ValueError("Excitations must have identical lengths.")
        dtype_ = np.float32
        dx, dy, dz = [conv.m_in(d).astype(dtype_) for d in self.d_cells]
        dx_h, dy_h, dz_h = [conv.m_in(d).astype(dtype_) for d in self.dh_cells]
        Nx, Ny, Nz = len(dx), len(dy), len(dz)
        dx_inv, dy_inv, dz_inv = 1 / dx[:, None, None], 1 / dy[None, :, None], 1 / dz[None, None, :]
        dx_h_inv, dy_h_inv, dz_h_inv = 1 / dx_h[:, None, None], 1 / dy_h[None, :, None], 1 / dz_h[None, None, :]
        dx1_h_inv = np.concatenate([dx_h_inv, [[[0]]]], axis=0)
        dy1_h_inv = np.concatenate([dy_h_inv, [[[0]]]], axis=1)
        dz1_h_inv = np.concatenate([dz_h_inv, [[[0]]]], axis=2)
        end = None if gpu else -1
        hs = 1 if gpu else 0
        Ca, Cb, Da, Db = self.Ca, self.Cb, self.Da, self.Db
        coefficients = dict(
            Ca_ex_y=Ca["ex_y"][:, 1:end, 1:end],
            Ca_ex_z=Ca["ex_z"][:, 1:end, 1:end],
            Cb_ex_y=Cb["ex_y"][:, 1:end, 1:end] * dy1_h_inv[:, :end],
            Cb_ex_z=-Cb["ex_z"][:, 1:end, 1:end] * dz1_h_inv[..., :end],
            Ca_ey_z=Ca["ey_z"][1:, :, 1:end],
            Ca_ey_x=Ca["ey_x"][1:, :, 1:end],
            Cb_ey_z=Cb["ey_z"][1:, :, 1:end] * dz1_h_inv[..., :end],
            Cb_ey_x=-Cb["ey_x"][1:, :, 1:end] * dx1_h_inv,
            Ca_ez_x=Ca["ez_x"][1:, 1:end, :],
            Ca_ez_y=Ca["ez_y"][1:, 1:end, :],
            Cb_ez_x=Cb["ez_x"][1:, 1:end, :] * dx1_h_inv,
            Cb_ez_y=-Cb["ez_y"][1:, 1:end, :] * dy1_h_inv[:, :end],
            Da_hx_y=Da["hx_y"][1:],
            Da_hx_z=Da["hx_z"][1:],
            Db_hx_y1=-Db["hx_y1"][1:] * dy_inv,
            Db_hx_y2=-Db["hx_y2"][1:] * dy_inv,
            Db_hx_z1=Db["hx_z1"][1:] * dz_inv,
            Db_hx_z2=Db["hx_z2"][1:] * dz_inv,
            Da_hy_z=Da["hy_z"][:, hs:],
            Da_hy_x=Da["hy_x"][:, hs:],
            Db_hy_z1=-Db["hy_z1"][:, hs:] * dz_inv,
            Db_hy_z2=-Db["hy_z2"][:, hs:] * dz_inv,
            Db_hy_x1=Db["hy_x1"][:, hs:] * dx_inv,
            Db_hy_x2=Db["hy_x2"][:, hs:] * dx_inv,
            Da_hz_x=Da["hz_x"][:, :, hs:],
            Da_hz_y=Da["hz_y"][:, :, hs:],
            Db_hz_x1=-Db["hz_x1"][:, :, hs:] * dx_inv,
            Db_hz_x2=-Db["hz_x2"][:, :, hs:] * dx_inv,
            Db_hz_y1=Db["hz_y1"][:, :, hs:] * dy_inv,
            Db_hz_y2=Db["hz_y2"][:, :, hs:] * dy_inv,
        )
        for k in coefficients:
            coefficients[k] = np.array(coefficients[k], order="C", dtype=dtype_)

        temp_mem_size = 0
        for s in self.fshape.values():
            temp_mem_size += 3 * np.prod((Nx,) + s[1:])
        temp_mem_size += (4 * (Ny + 1) * (Nz + 1)) * n_threads * 8
        mem = np.zeros(0 if gpu else temp_mem_size, dtype=dtype_)

        probes = []
        field_names = list(self.fshape.keys())
        for port in (self.ports + self.ports_inv):
            if port is None:
                continue
            idx, Vs_a, field, src = port["idx"], port["Vs_a"], port["field"], port["src"]
            if src is None:
                src = np.zeros(Nt, dtype=dtype_, order="C")
            idx_list = [list(np.arange(v.start, v.stop)) if isinstance(v, slice) else [v] for v in idx]
            Vs_a_flt = Vs_a.flatten()
            for j, idx_j in enumerate(itertools.product(*idx_list)):
                probes.append(dict(values=np.array(Vs_a_flt[j] * src, dtype=dtype_, order="C"),
                                   field=int(field_names.index(field)),
                                   idx=[int(i) for i in idx_j],
                                   is_source=int(port["src"] is not None)))
        for k, v in soft.items():
            probes.append(dict(values=np.array(v["src"], dtype=dtype_, order="C"),
                               field=int(field_names.index(v["field"])),
                               idx=[int(i) for i in v["index"]], is_source=1))
        for k, p in self.probes.items():
            probes.append(dict(values=np.zeros(Nt, dtype=dtype_, order="C"),
                               field=int(field_names.index(p["field"])),
                               idx=[int(i) for i in p["index"]], is_source=int(0)))

        monitors = []
        f_Ny = [self.Ny + 1, self.Ny, self.Ny + 1, self.Ny, self.Ny + 1, self.Ny]
        f_Nz = [self.Nz + 1, self.Nz + 1, self.Nz, self.Nz, self.Nz, self.Nz + 1]
        for k, m in self.monitors.items():
            n_m = int(Nt / m["n_step"]) + 1
            fi = field_names.index(m["field"])
            if m["axis"] == 0:
                m_shape = (Ny, Nz) if gpu else (f_Ny[fi], f_Nz[fi])
            elif m["axis"] == 1:
                m_shape = (Nx, Nz) if gpu else (self.Nx, f_Nz[fi])
            else:
                m_shape = (Nx, Ny) if gpu else (self.Nx, f_Ny[fi])
            cfg = dict(axis=int(m["axis"]), position=int(m["index"]), field=fi, n_step=int(m["n_step"]))
            if m["frequency"] is not None:
                frequency = m["frequency"]
                fs = (1 / (self.dt * m["n_step"]))
                omega = 2 * np.pi * (frequency / fs)
                cfg["values"] = np.zeros(((len(frequency),) + m_shape), dtype=np.complex64, order="C")
                cfg["dtft_phase"] = np.exp(-1j * omega[None] * np.arange(n_m)[:, None], dtype=np.complex64,
                                           order="C")
                cfg["n_frequencies"] = int(len(frequency))
            else:
                cfg["values"] = np.zeros(((n_m,) + m_shape), dtype=dtype_, order="C")
            monitors.append(cfg)
        return coefficients, probes, monitors, mem, Nx, Ny, Nz, Nt

    def unpack_results(self, probes, monitors, gpu: bool, Nt: int):
        """Move probe / monitor results back onto the model (rfnetwork/solver.py:1646-1698)."""
        for i, (k, m) in enumerate(self.monitors.items()):
            m_val = monitors[i]["values"]
            if m["axis"] in (1, 2) and m["field"] in ("hx", "ey", "ez"):
                m_val = np.pad(m_val, ((0, 0), (1, 0), (0, 0)))
            if gpu:
                if m["field"] in ("hy", "ex", "ez"):
                    if m["axis"] == 0:
                        m_val = np.pad(m_val, ((0, 0), (1, 0), (0, 0)))
                    if m["axis"] == 2:
                        m_val = np.pad(m_val, ((0, 0), (0, 0), (1, 0)))
                if m["field"] in ("hz", "ex", "ey"):
                    if m["axis"] == 0:
                        m_val = np.pad(m_val, ((0, 0), (0, 0), (1, 0)))
                    if m["axis"] == 1:
                        m_val = np.pad(m_val, ((0, 0), (0, 0), (1, 0)))
            self.monitors[k]["values"] = m_val
        src_v = [s["values"] for s in probes]
        probe_i = 0
        for port in (self.ports + self.ports_inv):
            if port is None:
                continue
            n = port["Vs_a"].size
            port["values"] = np.array(src_v[probe_i: probe_i + n]).reshape(port["Vs_a"].shape + (Nt,))
            probe_i += n
        for k, v in getattr(self, "soft_sources", {}).items():
            v["values"] = probes[probe_i]["values"]
            probe_i += 1
        for i, (k, p) in enumerate(self.probes.items()):
            self.probes[k]["values"] = probes[i + probe_i]["values"]
        self._solved = True

    def dft_series(self):
        """Port voltage / current series as weighted probe sums, for the on-device DFT.

        Returns ``(names, terms)``: names[s] is "V<i>" / "I<i>" (1-based
        port number) and each term is (series, probe index, weight), with the
        probe indices of ``pack_inputs``. The weights are those of
        get_sparameters (rfnetwork/solver.py:2482-2504): V = -dir * mean over
        the port width of sum(E * cell width), I = dir * sum(H * d).
        """
        names, terms = [], []
        offsets, off = [], 0
        for port in (self.ports + self.ports_inv):
            if port is None:
                offsets.append(None)
                continue
            offsets.append(off)
            off += port["Vs_a"].size
        n_soft = len(getattr(self, "soft_sources", {}))
        probe_index = {k: off + n_soft + i for i, k in enumerate(self.probes.keys())}
        for i, port in enumerate(self.ports):
            f_axis = dict(x=0, y=1, z=2)[port["field"][1]]
            idx = port["idx"]
            cell_w = conv.m_in(self.d_cells[f_axis][idx[f_axis]])
            shape = port["Vs_a"].shape
            n_w = int(np.prod([s for a, s in enumerate(shape) if a != f_axis]))
            s_v = len(names)
            names.append(f"V{i + 1}")
            for j in range(int(np.prod(shape))):
                f_pos = np.unravel_index(j, shape)[f_axis]
                terms.append((s_v, offsets[i] + j, -port["direction"] * float(cell_w[f_pos]) / n_w))
            s_i = len(names)
            names.append(f"I{i + 1}")
            prefix = f"port_{i + 1}"
            for k, p in self.probes.items():
                if k[:len(prefix)] == prefix:
                    terms.append((s_i, probe_index[k], port["direction"] * float(p["d"])))
        return names, terms

    def dft_omega(self, frequency: np.ndarray) -> np.ndarray:
        """Radians per time step, computed as utils.dtft does (fs = 1/dt)."""
        fs = 1 / self.dt
        return 2 * np.pi * (np.asarray(frequency) / fs)

    def solve(self, n_threads: int = 4, show_progress: bool = True, gpu: bool = True, frequency=None):
        """Run the time loop on the GPU (reference: rfnetwork/solver.py:1410-1700).

        Both ``gpu`` values run the B200 engine; the argument is kept so that
        reference scripts run unchanged. ``n_threads`` is accepted and unused.
        With ``frequency`` the port voltages and currents are also transformed
        on the device (FP64 running DFT); ``get_sparameters_device`` reads them.
        """
        from rfnetwork_b200 import cuda_func

        coefficients, probes, monitors, mem, Nx, Ny, Nz, Nt = self.pack_inputs(gpu=True, n_threads=n_threads)
        if frequency is None:
            cuda_func.solver_run_cu(coefficients, probes, monitors, mem, Nx, Ny, Nz, Nt, n_threads, 0)
            self.dft = None
        else:
            names, terms = self.dft_series()
            X = cuda_func.solver_run_dft(coefficients, probes, monitors, Nx, Ny, Nz, Nt, terms,
                                         self.dft_omega(frequency))
            self.dft = dict(frequency=np.asarray(frequency), names=names, X=X)
        self.last_run = cuda_func.last_run_info()
        self.unpack_results(probes, monitors, gpu=True, Nt=Nt)

    def get_sparameters_device(self, source_port: int = 1):
        """S-matrix column from the on-device DFT of the last ``solve(frequency=...)``.

        Same wave definitions as get_sparameters (rfnetwork/solver.py:2506-2514);
        returns (frequency, b, a=1).
        """
        self.check_solution()
        if getattr(self, "dft", None) is None:
            raise RuntimeError("solve() was run without frequency=...; no device DFT available.")
        names, X = self.dft["names"], self.dft["X"]
        nports = len(self.ports)
        Vp = np.array([X[names.index(f"V{i + 1}")] for i in range(nports)])
        Ip = np.array([X[names.index(f"I{i + 1}")] for i in range(nports)])
        r0 = np.array([p["r0"] for p in self.ports])[..., None]
        Ap = (Vp + r0 * Ip) / 2
        Bp = (Vp - r0 * Ip) / 2
        S = Bp / Ap[source_port - 1][None]
        return S.T[..., None]

    # ---------------------------------------------------------- results
    def line_probe_values(self, name: str) -> np.ndarray:
        """Raw probe series of a line probe (rfnetwork/solver.py:2425-2432)."""
        self.check_solution()
        return np.array([p["values"] for k, p in self.probes.items() if k[:len(name)] == name])

    def vi_probe_values(self, name: str) -> np.ndarray:
        """Sum of probe values times their signed widths (rfnetwork/solver.py:2434-2440)."""
        self.check_solution()
        return np.sum([p["values"] * p["d"] for k, p in self.probes.items() if k[:len(name)] == name], axis=0)

    def port_vi_series(self, i: int):
        """Time-domain voltage and current of port ``i`` (0-based), as get_sparameters forms them."""
        port = self.ports[i]
        field_idx, field, direction = port["idx"], port["field"], port["direction"]
        f_axis = dict(x=0, y=1, z=2)[field[1]]
        cell_w = conv.m_in(self.d_cells[f_axis][field_idx[f_axis]])
        b = [None] * 4
        b[f_axis] = slice(None)
        component_v = port["values"] * cell_w[tuple(b)]
        vp = (-direction) * np.sum(component_v, axis=f_axis).squeeze()
        if len(vp.shape) > 1:
            vp = np.mean(vp, axis=0)
        ip = self.vi_probe_values(f"port_{i + 1}")
        return vp, ip

    def get_sparameters(self, frequency: np.ndarray, source_port: int = 1, downsample: bool = False):
        """One column of the S matrix from port V and I (rfnetwork/solver.py:2442-2532).

        Returns an array of shape (frequency, b, a=1).
        """
        self.check_solution()
        nports, nf = len(self.ports), len(frequency)
        Vp = np.zeros((nports, nf), dtype=np.complex128)
        Ip = np.zeros((nports, nf), dtype=np.complex128)
        for i, port in enumerate(self.ports):
            vp, ip = self.port_vi_series(i)
            Vp[i] = dtft(vp, frequency, 1 / self.dt, downsample)
            Ip[i] = port["direction"] * dtft(ip, frequency, 1 / self.dt, downsample)
        r0 = np.array([p["r0"] for p in self.ports])[..., None]
        Ap = (Vp + r0 * Ip) / 2
        Bp = (Vp - r0 * Ip) / 2
        S = Bp / Ap[source_port - 1][None]
        return S.T[..., None]

    def get_total_monitor_data(self, name: str):
        """The three E components of an "e_total" monitor at common points of the
        monitor plane (rfnetwork/solver.py:2750-2802): each in-plane component
        averaged over its two neighbours along itself, the samples on the plane's
        edges dropped. Returns ``(values [3 (x, y, z), time, n1, n2], coords)``."""
        names = [f"{name}_{a}" for a in ("x", "y", "z")]
        if not all(n in self.monitors for n in names):
            raise ValueError(f"Monitor {name} does not contain data for all three field components.")
        m0 = self.monitors[names[0]]
        if m0["frequency"] is not None:
            raise NotImplementedError("Phasor monitors not implemented yet for total fields.")
        axis = m0["axis"]
        order = [a for a in range(3) if a != axis] + [axis]   # in-plane axes, then the normal
        data = [self.get_monitor_data(n) for n in names]
        e1, e2, e3 = [data[a][0] for a in order]
        cuts = ((slice(1, None), slice(1, -1)), (slice(1, -1), slice(1, None)), (slice(1, -1), slice(1, -1)))
        e1 = (e1[:, 1:, 1:-1] + e1[:, :-1, 1:-1]) / 2
        e2 = (e2[:, 1:-1, 1:] + e2[:, 1:-1, :-1]) / 2
        e3 = e3[:, 1:-1, 1:-1]
        comps = (e1, e2, e3)
        values = np.array([comps[order.index(a)] for a in range(3)])
        # coordinates of the x component's samples, as the reference labels the result
        vx, cx = data[0]
        cut = cuts[order.index(0)]
        coords = {"component": ("x", "y", "z"), "time": cx["time"]}
        for k, a in enumerate(order[:2]):
            coords["xyz"[a]] = cx["xyz"[a]][cut[k]]
        return values, coords

    def get_monitor_data(self, name: str):
        """Monitor samples with their coordinates (rfnetwork/solver.py:2703-2747).

        Returns ``(values, coords)``; coords maps ``time``/``frequency`` and
        the two in-plane axes to coordinate arrays (inches).
        """
        self.check_solution()
        m = self.monitors[name]
        axes = [0, 1, 2]
        axes.pop(m["axis"])
        coords = {}
        if m["frequency"] is not None:
            coords["frequency"] = m["frequency"]
        else:
            t_len = len(m["values"]) * self.dt * m["n_step"]
            coords["time"] = np.arange(0, t_len, self.dt * m["n_step"], dtype=np.float64)[:len(m["values"])]
        for a in axes:
            coords["xyz"[a]] = self.floc[m["field"]][a]
        return m["values"], coords
