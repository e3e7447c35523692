"""Numpy model of the engine's update arithmetic, driven by its material table.

Test helper: it replays what ``fdtd_step_kernel`` computes (unsplit update for
ordinary components, split update + soft sources for the components the table
flags as split, all in the
reference's GPU index space) from the table that the library's host compiler
produced. Comparing it with the CPU oracle checks the table compilation --
guards, x-end zeroing, split flags, probe shifts -- without a GPU.
"""
from __future__ import annotations

import numpy as np

FLAG_E, FLAG_H = 1, 2


def _f(rows, slot):
    return rows[:, slot].view(np.float32)


def run_model(ids, rows, cell_probes, probes, src, nt):
    """ids (nx,ny,nz) uint16, rows (R,32) uint32, probes: list of (field, x, y, z) shifted cells."""
    nx, ny, nz = ids.shape
    R = rows.copy()
    coef = {s: _f(R, s)[ids] for s in range(30)}
    flags = R[:, 30][ids]
    # component c (ex ey ez hx hy hz) stored as its split pair: flag bit 8 + c
    cs = [(flags & (1 << (8 + c))) != 0 for c in range(6)]
    f32 = np.float32
    E = [np.zeros(ids.shape, f32) for _ in range(3)]
    H = [np.zeros(ids.shape, f32) for _ in range(3)]
    Es = [np.zeros(ids.shape, f32) for _ in range(6)]
    Hs = [np.zeros(ids.shape, f32) for _ in range(6)]
    rec = np.zeros((len(probes), nt), f32)

    def fwd(a, axis):  # a[i+1] along axis, zero past the end
        out = np.zeros_like(a)
        sl_dst = [slice(None)] * 3
        sl_src = [slice(None)] * 3
        sl_dst[axis] = slice(0, -1)
        sl_src[axis] = slice(1, None)
        out[tuple(sl_dst)] = a[tuple(sl_src)]
        return out

    def bwd(a, axis):  # a[i-1] along axis, zero before the start
        out = np.zeros_like(a)
        sl_dst = [slice(None)] * 3
        sl_src = [slice(None)] * 3
        sl_dst[axis] = slice(1, None)
        sl_src[axis] = slice(0, -1)
        out[tuple(sl_dst)] = a[tuple(sl_src)]
        return out

    src_e = [(i, p) for i, p in enumerate(probes) if p[0] < 3]
    src_h = [(i, p) for i, p in enumerate(probes) if p[0] >= 3]
    for n in range(nt):
        hx, hy, hz = H
        d = {
            "hz_y": fwd(hz, 1) - hz, "hy_z": fwd(hy, 2) - hy, "hx_z": fwd(hx, 2) - hx,
            "hz_x": fwd(hz, 0) - hz, "hy_x": fwd(hy, 0) - hy, "hx_y": fwd(hx, 1) - hx,
        }
        dlist = [d["hz_y"], d["hy_z"], d["hx_z"], d["hz_x"], d["hy_x"], d["hx_y"]]
        # unsplit cells
        newE = []
        for c in range(3):
            ca, cb1, cb2 = coef[4 * c], coef[4 * c + 1], coef[4 * c + 3]
            newE.append(ca * E[c] + cb1 * dlist[2 * c] + cb2 * dlist[2 * c + 1])
        # split cells
        newEs = [coef[2 * s] * Es[s] + coef[2 * s + 1] * dlist[s] for s in range(6)]
        for i, (fld, x, y, z, is_src) in src_e:
            if is_src:
                v = src[i, n]
                newEs[2 * fld][x, y, z] += v
                newEs[2 * fld + 1][x, y, z] += v
        for c in range(3):
            tot = newEs[2 * c] + newEs[2 * c + 1]
            E[c] = np.where(cs[c], tot, newE[c]).astype(f32)
        for s in range(6):
            Es[s] = np.where(cs[s // 2], newEs[s], 0).astype(f32)
        ex, ey, ez = E
        g = [
            coef[14] * ez - coef[13] * bwd(ez, 1),   # hx_y
            coef[17] * ey - coef[16] * bwd(ey, 2),   # hx_z
            coef[20] * ex - coef[19] * bwd(ex, 2),   # hy_z
            coef[23] * ez - coef[22] * bwd(ez, 0),   # hy_x
            coef[26] * ey - coef[25] * bwd(ey, 0),   # hz_x
            coef[29] * ex - coef[28] * bwd(ex, 1),   # hz_y
        ]
        da = [coef[12], coef[15], coef[18], coef[21], coef[24], coef[27]]
        newH = [da[2 * c] * H[c] + g[2 * c] + g[2 * c + 1] for c in range(3)]
        newHs = [da[s] * Hs[s] + g[s] for s in range(6)]
        for i, (fld, x, y, z, is_src) in src_h:
            if is_src:
                v = src[i, n]
                c = fld - 3
                newHs[2 * c][x, y, z] += v
                newHs[2 * c + 1][x, y, z] += v
        for c in range(3):
            H[c] = np.where(cs[3 + c], newHs[2 * c] + newHs[2 * c + 1], newH[c]).astype(f32)
        for s in range(6):
            Hs[s] = np.where(cs[3 + s // 2], newHs[s], 0).astype(f32)
        for i, (fld, x, y, z, is_src) in enumerate(probes):
            rec[i, n] = (E + H)[fld][x, y, z]
    return rec


def shifted_probes(probe_dicts):
    """(field, x, y, z, is_source) after the Yee shift of solver_init_probes (solver.cpp:503-520)."""
    out = []
    for p in probe_dicts:
        f = int(p["field"])
        x, y, z = [int(v) for v in p["idx"]]
        if f in (1, 2, 3):
            x -= 1
        if f in (0, 2, 4):
            y -= 1
        if f in (0, 1, 5):
            z -= 1
        out.append((f, x, y, z, int(p.get("is_source", 0))))
    return out
