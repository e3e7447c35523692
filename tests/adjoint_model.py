"""FP64 numpy model of the engine's time stepping and of its discrete adjoint.

Test helper. ``forward`` replays the engine's update (the same arithmetic as
tests/kernel_model.py: unsplit update for ordinary cells, split update plus
soft sources for flagged cells, driven by the material table the library
compiled) in float64. ``adjoint`` runs the exact transpose of that linear
recursion backwards in time and returns the gradient of an objective with
respect to the E-update coefficients (Ca, Cb1, Cb2 of each component) of the
cells of a box. Finite differences of ``forward`` check ``adjoint``; the GPU
adjoint is checked against both.
"""
from __future__ import annotations

import numpy as np

FLAG_E, FLAG_H = 1, 2


def _f(rows, slot):
    return rows[:, slot].view(np.float32).astype(np.float64)


def fwd(a, axis):
    """a[i+1] along axis, zero past the end."""
    out = np.zeros_like(a)
    d = [slice(None)] * 3
    s = [slice(None)] * 3
    d[axis] = slice(0, -1)
    s[axis] = slice(1, None)
    out[tuple(d)] = a[tuple(s)]
    return out


def bwd(a, axis):
    """a[i-1] along axis, zero before the start."""
    out = np.zeros_like(a)
    d = [slice(None)] * 3
    s = [slice(None)] * 3
    d[axis] = slice(1, None)
    s[axis] = slice(0, -1)
    out[tuple(d)] = a[tuple(s)]
    return out


class Model:
    """Coefficients (float64, per cell) and split masks of a compiled table."""

    def __init__(self, ids, rows):
        self.shape = ids.shape
        self.coef = [_f(rows, s)[ids] for s in range(30)]
        flags = rows[:, 30][ids]
        self.es = (flags & FLAG_E) != 0
        self.hs = (flags & FLAG_H) != 0

    def with_coef(self, slot, values):
        m = Model.__new__(Model)
        m.shape, m.es, m.hs = self.shape, self.es, self.hs
        m.coef = list(self.coef)
        m.coef[slot] = values
        return m


def _diffs(H):
    hx, hy, hz = H
    # (dA, dB) per E component, the kernel's order (fdtd_kernels.cuh)
    return [(fwd(hz, 1) - hz, fwd(hy, 2) - hy),
            (fwd(hx, 2) - hx, fwd(hz, 0) - hz),
            (fwd(hy, 0) - hy, fwd(hx, 1) - hx)]


def _gterms(C, E):
    ex, ey, ez = E
    return [C[14] * ez - C[13] * bwd(ez, 1),   # hx_y
            C[17] * ey - C[16] * bwd(ey, 2),   # hx_z
            C[20] * ex - C[19] * bwd(ex, 2),   # hy_z
            C[23] * ez - C[22] * bwd(ez, 0),   # hy_x
            C[26] * ey - C[25] * bwd(ey, 0),   # hz_x
            C[29] * ex - C[28] * bwd(ex, 1)]   # hz_y


def step(model, probes, src, n, state):
    """One time step n of the engine's update: state = (E, H, Es, Hs) lists of
    arrays (3, 3, 6, 6) before the step; returns the state after it."""
    C, es, hs = model.coef, model.es, model.hs
    E, H, Es, Hs = state
    d = _diffs(H)
    newE, newEs = [], []
    for c in range(3):
        newE.append(C[4 * c] * E[c] + C[4 * c + 1] * d[c][0] + C[4 * c + 3] * d[c][1])
        newEs.append(C[4 * c] * Es[2 * c] + C[4 * c + 1] * d[c][0])
        newEs.append(C[4 * c + 2] * Es[2 * c + 1] + C[4 * c + 3] * d[c][1])
    for i, (fld, x, y, z, is_src) in enumerate(probes):
        if is_src and fld < 3:
            newEs[2 * fld][x, y, z] += src[i, n]
            newEs[2 * fld + 1][x, y, z] += src[i, n]
    E = [np.where(es, newEs[2 * c] + newEs[2 * c + 1], newE[c]) for c in range(3)]
    Es = [np.where(es, v, 0.0) for v in newEs]
    g = _gterms(C, E)
    da = [C[12], C[15], C[18], C[21], C[24], C[27]]
    newH = [da[2 * c] * H[c] + g[2 * c] + g[2 * c + 1] for c in range(3)]
    newHs = [da[s] * Hs[s] + g[s] for s in range(6)]
    for i, (fld, x, y, z, is_src) in enumerate(probes):
        if is_src and fld >= 3:
            c = fld - 3
            newHs[2 * c][x, y, z] += src[i, n]
            newHs[2 * c + 1][x, y, z] += src[i, n]
    H = [np.where(hs, newHs[2 * c] + newHs[2 * c + 1], newH[c]) for c in range(3)]
    Hs = [np.where(hs, v, 0.0) for v in newHs]
    return E, H, Es, Hs


def box_history(state, box):
    """E^n and the H differences (dA, dB) on the box, from the state before step n."""
    E, H = state[0], state[1]
    d = _diffs(H)
    sl = (slice(box[0], box[1]), slice(box[2], box[3]), slice(box[4], box[5]))
    return (np.array([E[c][sl] for c in range(3)]),
            np.array([[d[c][0][sl], d[c][1][sl]] for c in range(3)]))


def zero_state(shape):
    return ([np.zeros(shape) for _ in range(3)], [np.zeros(shape) for _ in range(3)],
            [np.zeros(shape) for _ in range(6)], [np.zeros(shape) for _ in range(6)])


def forward(model, probes, src, nt, box=None, states=None):
    """probes: (field, x, y, z, is_source) after the Yee shift; src: [P, nt].

    Returns rec [P, nt] and, with box = (x0, x1, y0, y1, z0, z1), the history
    of E^n and of the H differences (dA, dB) on the box for every step. With
    a dict `states`, the state before each step n in it is stored there."""
    state = zero_state(model.shape)
    rec = np.zeros((len(probes), nt))
    hist = [] if box is not None else None
    for n in range(nt):
        if states is not None and n in states:
            states[n] = state
        if hist is not None:
            hist.append(box_history(state, box))
        state = step(model, probes, src, n, state)
        E, H = state[0], state[1]
        for i, (fld, x, y, z, _) in enumerate(probes):
            rec[i, n] = (E + H)[fld][x, y, z]
    return rec, hist


def adjoint(model, probes, dJ_drec, box, hist):
    """Gradient of J with respect to (Ca, Cb1, Cb2) of each E component on the box.

    dJ_drec: [P, nt] = dJ / d rec. Returns g [3 components, 3 (Ca, Cb1, Cb2), *box shape]."""
    C, es, hs = model.coef, model.es, model.hs
    shp = model.shape
    nt = dJ_drec.shape[1]
    lE = [np.zeros(shp) for _ in range(3)]
    lEs = [np.zeros(shp) for _ in range(6)]
    lH = [np.zeros(shp) for _ in range(3)]
    lHs = [np.zeros(shp) for _ in range(6)]
    sl = (slice(box[0], box[1]), slice(box[2], box[3]), slice(box[4], box[5]))
    grad = np.zeros((3, 3) + tuple(b - a for a, b in zip(box[0::2], box[1::2])))
    da = [C[12], C[15], C[18], C[21], C[24], C[27]]
    for n in range(nt - 1, -1, -1):
        aET = [np.zeros(shp) for _ in range(3)]
        aHT = [np.zeros(shp) for _ in range(3)]
        for i, (fld, x, y, z, _) in enumerate(probes):
            (aET if fld < 3 else aHT)[fld % 3][x, y, z] += dJ_drec[i, n]
        # adjoints of the H^{n+1} states
        muH = [np.where(hs, 0.0, lH[c] + aHT[c]) for c in range(3)]
        muHs = [np.where(hs, lHs[s] + aHT[s // 2], 0.0) for s in range(6)]
        ag = [np.where(hs, muHs[s], muH[s // 2]) for s in range(6)]
        lH = [np.where(hs, 0.0, da[2 * c] * muH[c]) for c in range(3)]
        lHs = [np.where(hs, da[s] * muHs[s], 0.0) for s in range(6)]
        # H update -> E^{n+1} totals (transpose of the g terms)
        aET[2] += C[14] * ag[0] - fwd(C[13] * ag[0], 1)
        aET[1] += C[17] * ag[1] - fwd(C[16] * ag[1], 2)
        aET[0] += C[20] * ag[2] - fwd(C[19] * ag[2], 2)
        aET[2] += C[23] * ag[3] - fwd(C[22] * ag[3], 0)
        aET[1] += C[26] * ag[4] - fwd(C[25] * ag[4], 0)
        aET[0] += C[29] * ag[5] - fwd(C[28] * ag[5], 1)
        # adjoints of the E^{n+1} states
        muE = [np.where(es, 0.0, lE[c] + aET[c]) for c in range(3)]
        muEs = [np.where(es, lEs[s] + aET[s // 2], 0.0) for s in range(6)]
        E_n, d_n = hist[n]
        for c in range(3):
            m = muE[c][sl]
            grad[c, 0] += m * E_n[c]
            grad[c, 1] += m * d_n[c][0]
            grad[c, 2] += m * d_n[c][1]
        adA, adB = [], []
        for c in range(3):
            adA.append(np.where(es, C[4 * c + 1] * muEs[2 * c], C[4 * c + 1] * muE[c]))
            adB.append(np.where(es, C[4 * c + 3] * muEs[2 * c + 1], C[4 * c + 3] * muE[c]))
        lE = [np.where(es, 0.0, C[4 * c] * muE[c]) for c in range(3)]
        lEs = [np.where(es, C[4 * (s // 2) + 2 * (s % 2)] * muEs[s], 0.0) for s in range(6)]
        # E update -> H^n totals (transpose of the differences)
        aH = [np.zeros(shp) for _ in range(3)]
        aH[2] += bwd(adA[0], 1) - adA[0]
        aH[1] += bwd(adB[0], 2) - adB[0]
        aH[0] += bwd(adA[1], 2) - adA[1]
        aH[2] += bwd(adB[1], 0) - adB[1]
        aH[1] += bwd(adA[2], 0) - adA[2]
        aH[0] += bwd(adB[2], 1) - adB[2]
        lH = [np.where(hs, 0.0, lH[c] + aH[c]) for c in range(3)]
        lHs = [np.where(hs, lHs[s] + aH[s // 2], 0.0) for s in range(6)]
    return grad


def dft_objective(rec, probe, omega):
    """J = sum_f |sum_n rec[probe, n] e^{-j omega_f n}|^2 and dJ/drec."""
    n = np.arange(rec.shape[1])
    ph = np.exp(-1j * np.outer(omega, n))
    X = ph @ rec[probe]
    J = float(np.sum(np.abs(X) ** 2))
    g = np.zeros_like(rec)
    g[probe] = 2 * np.real(np.conj(X) @ ph)
    return J, g, X
