"""Near-field to far-field transform in numpy -- TEST INFRASTRUCTURE ONLY.

A restatement of the reference's postprocess_nf2ff
(rfnetwork/core/src/postprocess.cpp:130-505), which cannot be built here (it
needs the Eigen submodule that the checkout does not vendor). It takes the
arguments the reference binds as core_func.nf2ff (rfnetwork/solver.py:3014)
and fills ff_data["data"] in place, in complex128 arithmetic:
  * direction r^ = (sin th cos ph, sin th sin ph, cos th)        (postprocess.cpp:327-333)
  * per face, the cell positions (surf_pos, r_grid[0], r_grid[1]) in the
    face's axis order, phase exp(j beta r^ . r) times ds         (postprocess.cpp:370-431)
  * N_theta, N_phi from J, L_theta, L_phi from M                   (postprocess.cpp:433-480)
  * E_theta = (-j beta / 4 pi) (L_phi + eta0 N_theta),
    E_phi = (j beta / 4 pi) (L_theta - eta0 N_phi), eta0 = 376.730313 (postprocess.cpp:39, 490-497)
Used by tests/ to check the engine's fdtd_nf2ff; never by the product path.
"""
from __future__ import annotations

import numpy as np

ETA0 = 376.730313


def nf2ff(J_xyz, M_xyz, r_grid, ds_grid, surf_pos, ff_data) -> int:
    beta = np.asarray(ff_data["beta"], dtype=np.float64)
    th = np.asarray(ff_data["theta"], dtype=np.float64)[:, None]
    ph = np.asarray(ff_data["phi"], dtype=np.float64)[None, :]
    st, ct, sp, cp = np.sin(th), np.cos(th), np.sin(ph), np.cos(ph)
    uvw = (st * cp, st * sp, ct * np.ones_like(ph))
    out = np.zeros((2, len(beta), th.shape[0], ph.shape[1]), dtype=np.complex128)
    for f, b in enumerate(beta):
        N_t = np.zeros(out.shape[2:], dtype=np.complex128)
        N_p, L_t, L_p = N_t.copy(), N_t.copy(), N_t.copy()
        for axis in range(3):
            o0, o1 = [a for a in range(3) if a != axis]
            r0 = np.asarray(r_grid[axis][0], dtype=np.float64).ravel()
            r1 = np.asarray(r_grid[axis][1], dtype=np.float64).ravel()
            ds = np.real(np.asarray(ds_grid[axis])).astype(np.float64).ravel()
            for s in range(2):
                J = np.asarray(J_xyz[axis][s], dtype=np.complex128)[:, f].reshape(3, -1)
                M = np.asarray(M_xyz[axis][s], dtype=np.complex128)[:, f].reshape(3, -1)
                # r^ . r for every direction (rows) and cell (columns)
                rdot = (float(surf_pos[axis][s]) * uvw[axis][..., None] + r0 * uvw[o0][..., None]
                        + r1 * uvw[o1][..., None])
                w = np.exp(1j * b * rdot) * ds
                SJ = [w @ J[k] for k in range(3)]
                SM = [w @ M[k] for k in range(3)]
                N_t += SJ[0] * ct * cp + SJ[1] * ct * sp - SJ[2] * st
                N_p += -SJ[0] * sp + SJ[1] * cp
                L_t += SM[0] * ct * cp + SM[1] * ct * sp - SM[2] * st
                L_p += -SM[0] * sp + SM[1] * cp
        k = b / (4 * np.pi)
        out[0, f] = -1j * k * (L_p + ETA0 * N_t)
        out[1, f] = 1j * k * (L_t - ETA0 * N_p)
    ff_data["data"][...] = out
    return 0
