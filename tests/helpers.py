"""Shared helpers of the parity tests: run a model on the oracle or the engine
and compare the series the reference's post-processing uses."""
from __future__ import annotations

import copy

import numpy as np

from oracle import cpu_engine


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a))


def run_oracle(s, precision="f32", n_threads=None):
    """Run the CPU oracle on model ``s`` (CPU packing) and unpack onto a copy of ``s``."""
    s2 = copy.deepcopy(s)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s2.pack_inputs(gpu=False, n_threads=2)
    if precision == "f64":
        co = {k: v.astype(np.float64) for k, v in co.items()}
        for p in pr:
            p["values"] = p["values"].astype(np.float64)
        for m in mo:
            m["values"] = m["values"].astype(np.complex128 if np.iscomplexobj(m["values"]) else np.float64)
            if "dtft_phase" in m:
                m["dtft_phase"] = m["dtft_phase"].astype(np.complex128)
    cpu_engine.solver_run(co, pr, mo, mem, Nx, Ny, Nz, Nt, n_threads or cpu_engine.default_threads(), 0,
                          precision=precision)
    s2.unpack_results(pr, mo, gpu=False, Nt=Nt)
    return s2, np.array([p["values"] for p in pr])


def run_engine(s, frequency=None):
    s2 = copy.deepcopy(s)
    s2.solve(gpu=True, frequency=frequency)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s2.pack_inputs(gpu=True)
    # probe matrix in pack order, from the unpacked model
    rows = []
    for port in (s2.ports + s2.ports_inv):
        if port is None:
            continue
        rows.extend(port["values"].reshape(-1, Nt))
    for v in getattr(s2, "soft_sources", {}).values():
        rows.append(v["values"])
    for p in s2.probes.values():
        rows.append(p["values"])
    return s2, np.array(rows)


def derived_series(s):
    """Port V / I series and named probe sums, as get_sparameters / vi_probe_values form them."""
    out = {}
    for i in range(len(s.ports)):
        v, c = s.port_vi_series(i)
        out[f"V{i + 1}"] = v
        out[f"I{i + 1}"] = c
    groups = set()
    for k, p in s.probes.items():
        if k.startswith("port_"):
            continue
        head, _, tail = k.rpartition("_")
        if head and tail.isdigit():
            groups.add(head)
        else:
            out[k] = p["values"] * p["d"]
    for n in sorted(groups):
        out[n] = s.vi_probe_values(n + "_")
    return out
