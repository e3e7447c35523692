#!/usr/bin/env python
"""Throughput of the B200 FDTD engine on the bandwidth model.

Workload: 256 x 256 x 128 cells, 8-cell split-field PML on all faces, 64
seeded dielectric boxes, 4 lumped ports driven by a Gaussian pulse, 16 Ez
point probes and an FP64 running DFT at 51 frequencies of the port voltages,
port currents and probes; 5000 Yee time steps. One bench "step" is one full
simulation of that model (all 5000 time steps).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). ``value`` is Mcell-updates/s with the model
resident on the device (the time loop replayed as a CUDA graph on a stream of
this script, CUDA events around the K simulations, max over ranks);
``e2e`` is the same metric through the reference-facing call
(``rfnetwork_b200.cuda_func.solver_run_dft`` on host numpy arrays: coefficient
compilation, host-to-device copies, the run and the read-back of probes and
DFT inside the timed region). ``--impl reference`` times the CPU restatement
of the reference's threaded C++ solver on the host cores instead.

After the timed region, at N = 1, the line also carries its baselines and the
other workloads: ``cpu_baseline`` (the CPU restatement on a bounded sample),
``reference_cuda`` (the reference's own CUDA engine, solver.cu built from the
reference's sources, on the same model and steps: the drop-in comparison,
with the relative L2 difference of the two engines' probe series) and
``workloads`` (one timed run each of the microstrip solve uniform and graded,
the 64-simulation batch, the adjoint gradient and the design loop; each is also
``--workload NAME`` on its own).

With N > 1 (torchrun) every rank runs its own replica of the model (the
solver has no cross-GPU exchange); ``value`` is the sum over ranks.
"""
from __future__ import annotations

import argparse
import copy
import datetime
import json
import re
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

GRID = (256, 256, 128)
N_PML = 8
NT = 5000
N_FREQ = 51
WORKLOAD = "boxes 256x256x128, 8-cell PML, 64 dielectric boxes, 4 ports, 16 Ez probes, 51-freq DFT, 5000 steps"
METRIC = "Yee Mcell-updates/s"
UNIT = "Mcell-updates/s"
FALLBACK_HBM_GBS = 6650.0

SMI_FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--nt", type=int, default=NT, help="time steps per simulation")
    ap.add_argument("--e2e-steps", type=int, default=None, help="end-to-end calls timed (default: --steps)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reference-cuda", action="store_true", help="skip the reference CUDA engine comparison")
    ap.add_argument("--no-workloads", action="store_true", help="skip the other workloads after the timed region")
    ap.add_argument("--workload", choices=("boxes", "microstrip", "batch", "adjoint", "design"), default="boxes",
                    help="boxes: the bandwidth model (default); microstrip: the 64x64x48 microstrip with its "
                         "101-frequency S11/S21 (the case the reference runs on the CPU), solve time against the "
                         "CPU restatement of the reference engine; batch: 64 uneven simulations in one launch "
                         "per step against 64 sequential single-simulation runs; adjoint: forward + discrete "
                         "adjoint gradient of a 48x48x4 permittivity design against one forward solve; "
                         "design: Adam steps on 32 design variants, batched forward and batched adjoint")
    return ap.parse_args()


# --------------------------------------------------------------------- model

def bench_config(nt: int, world: int, n_series: int, n_probes: int) -> dict:
    """The workload's `config`, the same for both arms."""
    cells = GRID[0] * GRID[1] * GRID[2]
    interior = (GRID[0] - 2 * N_PML) * (GRID[1] - 2 * N_PML) * (GRID[2] - 2 * N_PML)
    # both time buffers of the 6 fields, the 16-bit index, 12 split halves per PML slab cell
    state = cells * (48 + 2) + (cells - interior) * 96
    return {"workload": WORKLOAD, "grid": list(GRID), "n_pml": N_PML, "time_steps": nt,
            "dft_frequencies": N_FREQ, "dft_series": n_series, "probes": n_probes,
            "l2": "inputs larger than L2 (fields, split-pair slab stores and index %.2f GB per replica)" % (state / 1e9),
            "parallelism": f"replicas{world}" if world > 1 else "single"}


def build_model(nt: int):
    from modelgen import configs
    return configs.boxes(n=GRID, n_pml=N_PML, nt=nt)


def dft_spec(s, pr):
    """Port V/I series of the S-parameter post-processing plus one series per point probe."""
    from modelgen import configs
    names, terms = s.dft_series()
    n_lead = len(pr) - len(s.probes)
    for i, k in enumerate(s.probes.keys()):
        if k.startswith("port_"):
            continue
        terms.append((len(names), n_lead + i, 1.0))
        names.append(k)
    omega = s.dft_omega(configs.boxes_frequencies(N_FREQ))
    return names, terms, omega


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic(variant: int, path: Path = None):
    """DRAM bytes of one step launch of this workload from the committed ncu
    summary (its line `traffic_bytes_per_launch (variant V): B`), or None."""
    tp = path or ROOT / "profiles" / "fdtd_step_stream_boxes256.md"
    if not tp.exists():
        return None
    m = re.search(r"traffic_bytes_per_launch \(variant %d\): (\d+)" % variant, tp.read_text())
    return int(m.group(1)) if m else None


# ------------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi samples of one GPU every 200 ms while the timed region runs."""

    def __init__(self, device_index: int):
        self.dev = str(device_index)
        try:  # the physical GPU behind a CUDA_VISIBLE_DEVICES remapping
            import torch
            u = str(torch.cuda.get_device_properties(device_index).uuid)
            self.dev = u if u.startswith("GPU-") else "GPU-" + u
        except Exception:
            pass
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"rfn_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={SMI_FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", self.dev], stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        if self.proc is None or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        try:
            self.path.unlink()
        except OSError:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------- ranks

class RankSync:
    """Barrier and max-over-ranks of one process per GPU (torchrun env).

    With world > 1 it joins the process group (NCCL on GPUs; gloo for the
    CPU tests of this logic) with a short timeout, so ranks that wait on a
    missing peer fail instead of hanging. With world == 1 it does nothing.
    Every rank must make the same calls in the same order."""

    def __init__(self, world: int, local_rank: int = 0, backend: str = "nccl", timeout_s: int = 600):
        import torch
        self.torch = torch
        self.dist = None
        self.cuda = backend == "nccl"
        if world > 1:
            import torch.distributed as dist
            kw = {"device_id": torch.device("cuda", local_rank)} if self.cuda else {}
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
            self.dist = dist

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()
        if self.cuda:
            self.torch.cuda.synchronize()

    def max(self, v: float) -> float:
        if self.dist is None:
            return v
        t = self.torch.tensor([v], dtype=self.torch.float64, device="cuda" if self.cuda else "cpu")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist is not None:
            self.dist.barrier()
            self.dist.destroy_process_group()
            self.dist = None


# ---------------------------------------------------------------- our arm

def run_ours(args, rank, world, local_rank):
    import torch
    from rfnetwork_b200 import _lib, cuda_func
    from modelgen import configs

    torch.cuda.set_device(local_rank)
    ranks = RankSync(world, local_rank)
    barrier, max_over_ranks = ranks.barrier, ranks.max

    nt = args.nt
    s = build_model(nt)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)
    names, terms, omega = dft_spec(s, pr)
    cells = Nx * Ny * Nz
    alg_bytes_step = configs.algorithmic_bytes((Nx, Ny, Nz), N_PML)

    # ---- device-resident arm: the model compiled once, the time loop replayed
    sim = _lib.Simulation(Nx, Ny, Nz)
    sim.set_coefficients(co)
    for p in pr:
        src = bool(p["is_source"])
        sim.add_probe(int(p["field"]), p["idx"], src, p["values"][:Nt] if src else None)
    sim.set_dft(terms, omega)
    stream = torch.cuda.Stream()
    sim.set_stream(stream.cuda_stream)
    for _ in range(max(args.warmup, 0)):
        sim.run_async(Nt)
        sim.synchronize()
    st = sim.stats()

    barrier()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    with ClockSampler(local_rank) as clk:
        evs[0].record(stream)
        for k in range(args.steps):
            sim.run_async(Nt)
            evs[k + 1].record(stream)
        sim.synchronize()
        torch.cuda.synchronize()
    barrier()
    per_sim_ms = [evs[k].elapsed_time(evs[k + 1]) for k in range(args.steps)]
    total_ms = max_over_ranks(sum(per_sim_ms))
    st = sim.stats()
    launches_per_sim = int(st["step_launches"] + st["dft_launches"])
    rec = sim.probe_values()
    finite = bool(np.isfinite(rec).all())
    sim.close()

    # ---- end to end through the reference-facing call, host arrays in and out
    e2e_steps = args.e2e_steps if args.e2e_steps is not None else args.steps
    e2e_s, info = 0.0, {}
    if e2e_steps > 0:
        pr_h = copy.deepcopy(pr)
        cuda_func.solver_run_dft(co, pr_h, mo, Nx, Ny, Nz, Nt, terms, omega)  # warm-up (driver, allocator)
        barrier()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            pr_h = copy.deepcopy(pr)
            cuda_func.solver_run_dft(co, pr_h, mo, Nx, Ny, Nz, Nt, terms, omega)
        torch.cuda.synchronize()
        e2e_s = max_over_ranks(time.perf_counter() - t0)
        info = cuda_func.last_run_info()

    ctx = {"co": co, "pr": pr, "shape": (Nx, Ny, Nz), "nt": Nt, "rec": rec, "e2e_s": e2e_s / max(e2e_steps, 1),
           "step_ms": statistics.fmean(per_sim_ms) / Nt}
    out = None
    if rank == 0:
        hbm, peak_kind = peaks()
        mean_sim_ms = statistics.fmean(per_sim_ms)
        step_ms = mean_sim_ms / Nt  # one step-kernel launch per time step (+ the DFT every 256 steps)
        achieved = alg_bytes_step / (step_ms * 1e-3) / 1e9
        traffic = profiled_traffic(st["variant"])
        value = world * cells * Nt * args.steps / (total_ms * 1e-3) / 1e6
        out = {
            "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded 64-box dielectric model (eps_r~U[1,10], sigma~U[0,0.05] S/m), "
                    "Gaussian-pulse ports",
            "config": bench_config(Nt, world, len(names), len(pr)),
            "step": f"one full simulation ({Nt} Yee time steps)",
            "kernel": {k: st[k] for k in ("variant", "tile_y", "stages", "zchunk", "grid", "n_tiles")},
            "autotune": {"ms": round(st["tune_ms"], 1), "trials": st["tune_trials"],
                         "when": "once per set of grid sizes per process, inside its first run (a warm-up run "
                                 "here); later runs take the cached shape"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                         "frac": round(achieved / hbm, 4), "traffic": traffic,
                         "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": alg_bytes_step,
                         "launch_ms": round(step_ms, 5),
                         "launch_ms_source": "CUDA events over the timed simulations / time steps"},
            "e2e": None if e2e_steps <= 0 else {
                "value": round(world * cells * Nt * e2e_steps / e2e_s / 1e6, 1), "unit": UNIT,
                "h2d_bytes_per_step": int(info.get("h2d_bytes", 0)),
                "d2h_bytes_per_step": int(info.get("d2h_bytes", 0)),
                "s_per_step": round(e2e_s / e2e_steps, 3), "call": "cuda_func.solver_run_dft",
                "compile_ms": round(float(info.get("compile_ms", 0.0)), 1)},
            "gpu_launches": launches_per_sim * args.steps,
            "clocks": clk.summary(),
            "finite": finite,
        }
    ranks.close()
    return out, ctx


# ----------------------------------------------------------- CPU baseline

def cpu_sample(nt_sample: int, n_threads: int):
    """Run the CPU restatement of the reference solver on the full grid for nt_sample steps.

    Returns (Mcell-updates/s, seconds)."""
    from oracle import cpu_engine
    s = build_model(nt_sample)
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=False)
    cpu_engine.build()
    t0 = time.perf_counter()
    cpu_engine.solver_run(co, pr, mo, mem, Nx, Ny, Nz, Nt, n_threads, 0)
    dt = time.perf_counter() - t0
    return Nx * Ny * Nz * Nt / dt / 1e6, dt


def sample_steps(n_threads: int, seconds: float = 10.0) -> int:
    """Time steps of the full grid that take about `seconds` on the CPU (8..256)."""
    v, _ = cpu_sample(2, n_threads)
    cells = GRID[0] * GRID[1] * GRID[2]
    return int(min(256, max(8, seconds * v * 1e6 / cells)))


def host_cpu() -> str:
    """The host CPU's model name (/proc/cpuinfo), or the platform's processor string."""
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.lower().startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def cpu_baseline_entry():
    from oracle import cpu_engine
    n = cpu_engine.default_threads()
    nt_sample = sample_steps(n)
    v, dt = cpu_sample(nt_sample, n)
    # the reference solve()'s default n_threads (rfnetwork/solver.py:1410), on a short sample
    v4, dt4 = cpu_sample(8, 4)
    return {"value": round(v, 2), "unit": UNIT, "cores": n, "kind": "port",
            "sample": f"{nt_sample} time steps of the {GRID[0]}x{GRID[1]}x{GRID[2]} model ({dt:.1f} s)",
            "host": {"cpu": host_cpu(), "nproc": os.cpu_count()},
            "at_reference_default_threads": {"value": round(v4, 2), "cores": 4,
                                             "sample": f"8 time steps of the same model ({dt4:.1f} s)"}}


def run_reference(args, rank, world):
    """CPU restatement of the reference's threaded C++ solver (solver.cpp), all usable host threads.

    Each step is a bounded sample of the workload (a few dozen time steps of the
    full grid); ``ms_per_step`` is the measured wall time of one sample."""
    if rank != 0:
        return None
    from oracle import cpu_engine
    from modelgen import configs
    n = cpu_engine.default_threads()
    for _ in range(max(args.warmup, 0)):
        cpu_sample(2, n)
    nt_sample = sample_steps(n)
    vals, secs = [], []
    for _ in range(args.steps):
        v, dt = cpu_sample(nt_sample, n)
        vals.append(v)
        secs.append(dt)
    value = statistics.fmean(vals)
    s = build_model(2)
    co, pr, *_ = s.pack_inputs(gpu=True)
    names, _terms, _omega = dft_spec(s, pr)
    return {
        "impl": "reference", "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(statistics.fmean(secs) * 1e3, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded 64-box dielectric model (eps_r~U[1,10], sigma~U[0,0.05] S/m), "
                "Gaussian-pulse ports",
        "config": bench_config(args.nt, world, len(names), len(pr)),
        "step": f"a sample of {nt_sample} time steps of the full grid (ms_per_step is its measured wall time)",
        "cpu_baseline": {"value": round(value, 2), "unit": UNIT, "cores": n, "kind": "port",
                         "sample": f"{nt_sample} time steps of the full grid per step"},
        "e2e": {"value": round(value, 2), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def reference_cuda_entry(ctx):
    """The drop-in comparison: the reference's own CUDA engine (rfnetwork/core/src/solver.cu,
    built unmodified from the reference's sources into oracle/_ref) on the same packed
    model and the same number of steps, outside the timed region. Wall time of its
    solver_run_cu (allocation, copies, four launches per step, read-back), its kernels'
    device time per step from a CUPTI trace, and the relative L2 difference between its
    probe series and this engine's end-to-end probe series."""
    try:
        from oracle import ref_cuda
        if not ref_cuda.available():
            return {"unavailable": "oracle/_ref/libref_cuda.so not built (needs the reference checkout at build time)"}
        import torch
        from torch.profiler import ProfilerActivity, profile
        co, pr, (Nx, Ny, Nz), nt = ctx["co"], ctx["pr"], ctx["shape"], ctx["nt"]
        mem = np.zeros(0, np.float32)
        ref_cuda.solver_run_cu(co, copy.deepcopy(pr), [], mem, Nx, Ny, Nz, nt, 0, 0)  # warm-up
        pr_ref = copy.deepcopy(pr)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ref_cuda.solver_run_cu(co, pr_ref, [], mem, Nx, Ny, Nz, nt, 0, 0)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        nt_prof = min(nt, 200)
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            ref_cuda.solver_run_cu(co, copy.deepcopy(pr), [], mem, Nx, Ny, Nz, nt_prof, 0, 0)
        kern_us = sum(e.time_range.elapsed_us() for e in prof.events() if "update_kernel" in e.name)
        ref_step_ms = kern_us / nt_prof / 1e3
        ref_rec = np.stack([p["values"][:nt] for p in pr_ref])
        ours = ctx["rec"]
        rel = float(np.linalg.norm(ours - ref_rec) / np.linalg.norm(ref_rec))
        cells = Nx * Ny * Nz
        return {
            "kind": "reference", "engine": "rfnetwork/core/src/solver.cu solver_run_cu, unmodified, sm_100a",
            "time_steps": nt, "wall_s": round(wall, 3), "e2e_mcell_updates_per_s": round(cells * nt / wall / 1e6, 1),
            "kernel_ms_per_step": round(ref_step_ms, 4),
            "kernel_mcell_updates_per_s": round(cells / ref_step_ms / 1e3, 1),
            "kernel_timing": f"CUPTI kernel trace (torch.profiler) over {nt_prof} steps",
            "ours_e2e_s": round(ctx["e2e_s"], 3), "ours_step_ms": round(ctx["step_ms"], 4),
            "e2e_speedup": round(wall / ctx["e2e_s"], 2), "step_speedup": round(ref_step_ms / ctx["step_ms"], 2),
            "probe_rel_l2_vs_ours": rel,
        }
    except Exception as e:  # a baseline, not the measurement: report why it is missing
        return {"unavailable": f"{type(e).__name__}: {e}"}


def reference_cuda_sequential(packed, nt, recs, cells_total):
    """The batch's first members run one after another through the reference's own CUDA
    engine (rfnetwork/core/src/solver.cu solver_run_cu, built unmodified into oracle/_ref:
    allocation, copies, four kernel launches per step, read-back), as a user of the
    reference runs them; wall time per member, scaled to the whole batch by the members'
    cell-steps. Outside every timed region; a baseline, not the measurement."""
    try:
        from oracle import ref_cuda
        if not ref_cuda.available():
            return {"unavailable": "oracle/_ref/libref_cuda.so not built (needs the reference checkout at build time)"}
        import torch
        mem = np.zeros(0, np.float32)
        co, pr, (Nx, Ny, Nz) = packed[0]
        ref_cuda.solver_run_cu(co, copy.deepcopy(pr), [], mem, Nx, Ny, Nz, nt, 0, 0)  # warm-up
        wall, cells, worst = 0.0, 0, 0.0
        for (co, pr, (Nx, Ny, Nz)), ours in zip(packed, recs):
            pr_ref = copy.deepcopy(pr)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ref_cuda.solver_run_cu(co, pr_ref, [], mem, Nx, Ny, Nz, nt, 0, 0)
            torch.cuda.synchronize()
            wall += time.perf_counter() - t0
            cells += Nx * Ny * Nz
            ref_rec = np.stack([p["values"][:nt] for p in pr_ref])
            worst = max(worst, float(np.linalg.norm(ours[:, :nt] - ref_rec) / np.linalg.norm(ref_rec)))
        return {"members": len(packed), "time_steps": nt, "wall_s": round(wall, 3),
                "sims_per_s": round(len(packed) / wall, 3),
                "ms_per_batch": round(wall * 1e3 * cells_total / cells, 2),
                "mcell_updates_per_s": round(cells * nt / wall / 1e6, 1),
                "probe_rel_l2_vs_ours_max": worst,
                "how": "wall time of solver_run_cu per member (allocation, copies, four launches per step, "
                       "read-back); ms_per_batch scales the sample to all members by their cells"}
    except Exception as e:  # a baseline, not the measurement: report why it is missing
        return {"unavailable": f"{type(e).__name__}: {e}"}


def workloads_entry(args, local_rank):
    """One timed run of each other workload (N = 1; three gradient evaluations for the
    adjoint, whose single wall-time samples vary most), summarised."""
    import argparse as _ap
    out = {}
    base = dict(vars(args))
    base.update(steps=1, warmup=1, nt=NT, no_cpu_baseline=True)

    def ns(**kw):
        d = dict(base)
        d.update(kw)
        return _ap.Namespace(**d)

    def keep(line, keys):
        return {k: line[k] for k in keys if k in line}

    common = ("value", "unit", "ms_per_step", "e2e", "cpu_baseline", "gpu_launches")
    for name, fn, kw, keys in (
            ("microstrip", run_microstrip, dict(no_cpu_baseline=False), common),
            ("microstrip_graded", run_microstrip, dict(graded=True), common),
            ("batch", run_batch, {}, ("value", "unit", "ms_per_step", "sequential", "batched_over_sequential",
                                      "sequential_plain_launches", "batched_over_sequential_plain_launches",
                                      "sequential_reference_cuda", "batched_over_sequential_reference_cuda",
                                      "mcell_updates_per_s", "bit_identical_to_sequential", "gpu_launches")),
            ("adjoint", run_adjoint, dict(steps=3), ("value", "unit", "ms_per_step", "forward_s", "gradient_over_forward",
                                          "device", "recorded_history", "checkpoints_every_32",
                                          "gradients_bit_identical_across_modes", "gpu_launches")),
            ("design", run_design, {}, ("value", "unit", "ms_per_step", "device", "recorded_history",
                                        "sequential", "batched_over_sequential", "gpu_launches"))):
        t0 = time.perf_counter()
        try:
            line = fn(ns(**kw), 0, 1, local_rank)
            out[name] = dict(keep(line, keys), config=line["config"]["workload"] if "config" in line else None,
                             wall_s=round(time.perf_counter() - t0, 1))
        except Exception as e:
            out[name] = {"error": f"{type(e).__name__}: {e}"}
    u, g = out.get("microstrip", {}), out.get("microstrip_graded", {})
    if "value" in u and "value" in g:
        # cell-update throughput of the non-uniform mesh against the uniform one
        g["mcell_rate_vs_uniform"] = round(g["value"] / u["value"], 3)
    return out


# ------------------------------------------------------ microstrip workload

def run_microstrip(args, rank, world, local_rank):
    """64x64x48 microstrip, 10-cell PML on six faces, 2000 steps, two 50-ohm ports, S11 and
    S21 at 101 frequencies from the device DFT: the reference's small case, which it runs on
    the CPU. One step is one full solve. Device time (CUDA events), end to end through
    cuda_func.solver_run_dft with host arrays, and the CPU restatement of the reference
    engine on the same model beside it (rank 0, N = 1)."""
    import torch
    from rfnetwork_b200 import _lib, cuda_func
    from modelgen import configs

    torch.cuda.set_device(local_rank)
    ranks = RankSync(world, local_rank)
    nt = args.nt if args.nt != NT else 2000
    graded = bool(getattr(args, "graded", False))
    s = configs.microstrip(nt=nt, graded=graded)
    f = configs.microstrip_frequencies()
    co, pr, mo, mem, Nx, Ny, Nz, Nt = s.pack_inputs(gpu=True)
    names, terms = s.dft_series()
    omega = s.dft_omega(f)
    cells = Nx * Ny * Nz
    sim = _lib.Simulation(Nx, Ny, Nz)
    sim.set_coefficients(co)
    for p in pr:
        src = bool(p["is_source"])
        sim.add_probe(int(p["field"]), p["idx"], src, p["values"][:Nt] if src else None)
    sim.set_dft(terms, omega)
    stream = torch.cuda.Stream()
    sim.set_stream(stream.cuda_stream)
    for _ in range(max(args.warmup, 0)):
        sim.run_async(Nt)
        sim.synchronize()
    ranks.barrier()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    evs[0].record(stream)
    for k in range(args.steps):
        sim.run_async(Nt)
        evs[k + 1].record(stream)
    sim.synchronize()
    torch.cuda.synchronize()
    ranks.barrier()
    dev_ms = ranks.max(sum(evs[k].elapsed_time(evs[k + 1]) for k in range(args.steps)) / args.steps)
    st = sim.stats()
    sim.close()
    pr_h = copy.deepcopy(pr)
    cuda_func.solver_run_dft(co, pr_h, mo, Nx, Ny, Nz, Nt, terms, omega)  # warm-up
    ranks.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        pr_h = copy.deepcopy(pr)
        cuda_func.solver_run_dft(co, pr_h, mo, Nx, Ny, Nz, Nt, terms, omega)
    torch.cuda.synchronize()
    e2e_s = ranks.max((time.perf_counter() - t0) / args.steps)
    info = cuda_func.last_run_info()
    ranks.close()
    if rank != 0:
        return None
    out = {
        "metric": METRIC, "value": round(world * cells * Nt / (dev_ms * 1e-3) / 1e6, 1), "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dev_ms, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: microstrip on a PEC ground plane, Gaussian-modulated port excitation",
        "config": {"workload": f"microstrip 64x64x48{' graded mesh (2-cell widths above the strip and '
                               'towards the y sides)' if graded else ''}, 10-cell PML, {Nt} steps, 2 ports, "
                               f"101-freq S11/S21", "grid": [Nx, Ny, Nz],
                   "cells": cells, "time_steps": Nt, "step": "one full solve",
                   "kernel": {k: st[k] for k in ("variant", "tile_y", "stages", "zchunk", "grid", "n_tiles")}},
        "e2e": {"value": round(world * cells * Nt / e2e_s / 1e6, 1), "unit": UNIT,
                "h2d_bytes_per_step": int(info.get("h2d_bytes", 0)),
                "d2h_bytes_per_step": int(info.get("d2h_bytes", 0)),
                "s_per_step": round(e2e_s, 4), "call": "cuda_func.solver_run_dft"},
        "gpu_launches": int(st["step_launches"] + st["dft_launches"]) * args.steps,
    }
    if world == 1 and not args.no_cpu_baseline:
        from oracle import cpu_engine
        n_thr = cpu_engine.default_threads()
        cpu_engine.build()
        c_co, c_pr, c_mo, c_mem, cNx, cNy, cNz, cNt = s.pack_inputs(gpu=False)
        t0 = time.perf_counter()
        cpu_engine.solver_run(c_co, c_pr, c_mo, c_mem, cNx, cNy, cNz, cNt, n_thr, 0)
        cpu_s = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": round(cells * Nt / cpu_s / 1e6, 2), "unit": UNIT, "cores": n_thr,
                               "kind": "port", "sample": f"the full {Nt}-step solve ({cpu_s:.2f} s)"}
    return out


# ------------------------------------------------------------ batched workload

BATCH_SIMS = 64
BATCH_NT = 3000
BATCH_FREQ = 21
BATCH_REF_SAMPLE = 8   # members the reference CUDA engine runs one after another


def run_batch(args, rank, world, local_rank):
    """64 simulations with seeded axes U{32..160}, 8-cell PML, 8 boxes, one Gaussian point
    source, 4 Ez probes, 21-frequency DFT each; stepped together (fdtd_batch_run: one step
    launch per time step for all of them, the time loop as one CUDA graph) and one after
    another (fdtd_run per simulation). Each rank runs its own copy."""
    import torch
    from rfnetwork_b200 import _lib
    from modelgen import configs

    torch.cuda.set_device(local_rank)
    ranks = RankSync(world, local_rank)
    nt = args.nt if args.nt != NT else BATCH_NT
    sims, cells, packed = [], 0, []
    for i in range(BATCH_SIMS):
        m = configs.batch_member(3, i, nt=nt)
        co, pr, mo, mem, Nx, Ny, Nz, Nt = m.pack_inputs(gpu=True)
        if i < BATCH_REF_SAMPLE:
            packed.append((co, copy.deepcopy(pr), (Nx, Ny, Nz)))
        sim = _lib.Simulation(Nx, Ny, Nz)
        sim.set_coefficients(co)
        for p in pr:
            src = bool(p["is_source"])
            sim.add_probe(int(p["field"]), p["idx"], src, p["values"][:Nt] if src else None)
        f = np.linspace(1e9, 20e9, BATCH_FREQ)
        sim.set_dft([(k, k, 1.0) for k in range(len(pr))], 2 * np.pi * f * float(m.dt))
        sims.append(sim)
        cells += Nx * Ny * Nz
    batch = _lib.Batch(sims)
    for _ in range(max(args.warmup, 1)):
        batch.run(nt)
    t_batch = []
    for _ in range(args.steps):
        batch.run(nt)
        t_batch.append(batch.stats()["last_run_ms"])
    recs = [s.probe_values().copy() for s in sims]
    # the same simulations one after another, each through its own run
    for s in sims:
        s.run(nt)
    t_seq = []
    for _ in range(args.steps):
        tot = 0.0
        for s in sims:
            s.run(nt)
            tot += s.stats()["last_run_ms"]
        t_seq.append(tot)
    same = all(np.array_equal(s.probe_values(), r) for s, r in zip(sims, recs))
    # and one after another with the plain kernel, every step launched from the
    # host (no graph), as the reference's engine runs a simulation
    t_plain = []
    for s in sims:
        s.set_kernel(0)
        s.set_graph(False)
        s.run(nt)
    for _ in range(args.steps):
        tot = 0.0
        for s in sims:
            s.run(nt)
            tot += s.stats()["last_run_ms"]
        t_plain.append(tot)
    same = same and all(np.array_equal(s.probe_values(), r) for s, r in zip(sims, recs))
    ref_seq = reference_cuda_sequential(packed, nt, recs[:len(packed)], cells) if rank == 0 else None
    st = batch.stats()
    batch.close()
    for s in sims:
        s.close()
    # each rank runs its own copy: the job takes as long as the slowest rank
    ms_b, ms_s, ms_p = (ranks.max(statistics.fmean(t)) for t in (t_batch, t_seq, t_plain))
    ranks.close()
    if rank != 0:
        return None
    return {
        "metric": "batched sims/s", "value": round(world * BATCH_SIMS / (ms_b * 1e-3), 3), "unit": "sims/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_b, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: seeded uneven grids with dielectric boxes and a Gaussian point source",
        "config": {"workload": f"batch of {BATCH_SIMS} sims, axes U{{32..160}}, 8-cell PML, {nt} steps, "
                               f"{BATCH_FREQ}-freq DFT", "cells_total": cells, "time_steps": nt,
                   "step": "one batched run of all simulations",
                   "kernel": {k: st[k] for k in ("variant", "tile_y", "stages", "zchunk", "grid", "n_tiles")}},
        "sequential": {"value": round(world * BATCH_SIMS / (ms_s * 1e-3), 3), "unit": "sims/s",
                       "ms_per_step": round(ms_s, 2)},
        "batched_over_sequential": round(ms_s / ms_b, 3),
        "sequential_plain_launches": {"value": round(world * BATCH_SIMS / (ms_p * 1e-3), 3), "unit": "sims/s",
                                      "ms_per_step": round(ms_p, 2),
                                      "how": "fdtd_run per simulation, plain kernel, every step launched "
                                             "from the host (no CUDA graph); device time incl. launch gaps"},
        "batched_over_sequential_plain_launches": round(ms_p / ms_b, 3),
        "sequential_reference_cuda": ref_seq,
        "batched_over_sequential_reference_cuda": (round(ref_seq["ms_per_batch"] / ms_b, 3)
                                                   if ref_seq and "ms_per_batch" in ref_seq else None),
        "mcell_updates_per_s": round(world * cells * nt / (ms_b * 1e-3) / 1e6, 1),
        "bit_identical_to_sequential": same,
        "gpu_launches": int(st["step_launches"] + st["dft_launches"]) * args.steps,
    }


# ---------------------------------------------------------- adjoint workload

def run_adjoint(args, rank, world, local_rank):
    """128x128x96 microstrip, 10-cell PML, 4000 steps; a 48x48x4-cell design block above
    the strip with eps_r = 1 + 9 sigmoid(theta), theta ~ N(0, 1) (seed 4); J = sum over
    11 frequencies (8-12 GHz) of |DFT of the output Ez probe|^2; checkpoints every 64 steps.
    One step = one gradient evaluation (forward with checkpoints + adjoint sweep). The same
    gradient with the box history recorded instead of checkpoints is reported beside it."""
    import torch
    from modelgen import configs
    from rfnetwork_b200.adjoint import FDTDDesign

    torch.cuda.set_device(local_rank)
    ranks = RankSync(world, local_rank)
    nt = args.nt if args.nt != NT else 4000
    s = configs.microstrip(n=(128, 128, 96), n_pml=10, nt=nt)
    co, pr, *_ = s.pack_inputs(gpu=True)
    omega = 2 * np.pi * np.linspace(8e9, 12e9, 11) * float(s.dt)
    box = (40, 88, 40, 88, 25, 29)
    gen = torch.Generator().manual_seed(4)
    theta = torch.randn(48, 48, 4, dtype=torch.float64, generator=gen)

    def measure(design):
        def grad_eval():
            t = theta.clone().requires_grad_(True)
            J = (design(1 + 9 * torch.sigmoid(t)).abs() ** 2).sum()
            J.backward()
            return float(J.detach()), t.grad

        for _ in range(max(args.warmup, 1)):
            grad_eval()
        t_grad, fwd_dev, adj_dev = [], [], []
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            J, g = grad_eval()
            torch.cuda.synchronize()
            t_grad.append(time.perf_counter() - t0)
            st = design.sim.stats()
            fwd_dev.append(st["last_run_ms"] / 1e3)
            adj_dev.append(st["adjoint_ms"] / 1e3)
        design.forward_only(1 + 9 * torch.sigmoid(theta))
        t_fwd, plain_dev = [], []
        for _ in range(args.steps):   # the plain forward solve of the same design, for the ratio
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            design.forward_only(1 + 9 * torch.sigmoid(theta))
            torch.cuda.synchronize()
            t_fwd.append(time.perf_counter() - t0)
            plain_dev.append(design.sim.stats()["last_run_ms"] / 1e3)
        st = design.sim.stats()
        design.close()
        tg, tf = ranks.max(statistics.fmean(t_grad)), ranks.max(statistics.fmean(t_fwd))
        dev_grad = statistics.fmean(fwd_dev) + statistics.fmean(adj_dev)
        dev_plain = statistics.fmean(plain_dev)
        return {
            "value": round(world / tg, 4), "ms_per_step": round(tg * 1e3, 1), "J": J,
            "forward_s": round(tf, 3), "gradient_over_forward": round(tg / tf, 3),
            "device": {"forward_for_gradient_s": round(statistics.fmean(fwd_dev), 4),
                       "adjoint_s": round(statistics.fmean(adj_dev), 4), "plain_forward_s": round(dev_plain, 4),
                       "gradient_over_forward": round(dev_grad / dev_plain, 3),
                       "adjoint_launches": st["adjoint_launches"]},
            "gpu_launches": int(st["step_launches"] + st["adjoint_launches"]),
            "grad": g.detach().clone(),
        }

    ck = measure(FDTDDesign(s, box, [(0, len(pr) - 1, 1.0)], omega, checkpoint_every=64))
    ck32 = measure(FDTDDesign(s, box, [(0, len(pr) - 1, 1.0)], omega, checkpoint_every=32))
    rec = measure(FDTDDesign(s, box, [(0, len(pr) - 1, 1.0)], omega))
    same = bool(torch.equal(ck.pop("grad"), rec["grad"]) and torch.equal(ck32.pop("grad"), rec.pop("grad")))
    ranks.close()
    if rank != 0:
        return None
    return {
        "metric": "grad evals/s", "value": ck["value"], "unit": "gradient evaluations/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ck["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 fields, f64 accumulators",
        "data": "synthetic: microstrip background, seeded theta",
        "config": {"workload": f"adjoint: 128x128x96, 10-cell PML, {nt} steps, 48x48x4 design, 11 freqs, "
                               "checkpoints every 64", "time_steps": nt, "design_cells": 48 * 48 * 4,
                   "step": "one gradient evaluation (forward with checkpoints + adjoint), wall time"},
        "forward_s": ck["forward_s"], "gradient_over_forward": ck["gradient_over_forward"], "device": ck["device"],
        "J": ck["J"], "gpu_launches": ck["gpu_launches"],
        "recorded_history": {k: rec[k] for k in ("value", "ms_per_step", "forward_s", "gradient_over_forward",
                                                   "device", "J")},
        "checkpoints_every_32": {k: ck32[k] for k in ("value", "ms_per_step", "gradient_over_forward", "device")},
        "replay": "each replayed step runs the tiles within reach of the design box (the steps left in its "
                  "segment, in cells)",
        "gradients_bit_identical_across_modes": same,
    }


# ---------------------------------------------------- batched design workload

def run_design(args, rank, world, local_rank):
    """32 variants of a 96x96x64 microstrip (10-cell PML, 3000 steps), each with its own
    32x32x4-cell design block above the strip, eps_r = 1 + 9 sigmoid(theta), theta ~ N(0, 1)
    (seed 5); J_i = sum over 5 frequencies (8-12 GHz) of |DFT of the output Ez probe|^2.
    One step = one Adam step (lr 0.05) on all 32 designs: a batched forward solve with state
    snapshots every ~sqrt(nt) steps, a batched adjoint sweep that replays the segments of all
    variants together, the optimizer update. Beside it: the same Adam step with the box
    histories recorded instead (no replay), and the 32 gradients one after another through
    FDTDDesign with the same checkpoints."""
    import math
    import torch
    from modelgen import configs
    from rfnetwork_b200.adjoint import FDTDDesign, FDTDDesignBatch

    torch.cuda.set_device(local_rank)
    ranks = RankSync(world, local_rank)
    nt = args.nt if args.nt != NT else 3000
    n_var = 32
    every = max(1, round(math.sqrt(nt)))
    s = configs.microstrip(n=(96, 96, 64), n_pml=10, nt=nt)
    co, pr, *_ = s.pack_inputs(gpu=True)
    omega = 2 * np.pi * np.linspace(8e9, 12e9, 5) * float(s.dt)
    box = (32, 64, 32, 64, 22, 26)
    terms = [(0, len(pr) - 1, 1.0)]
    gen = torch.Generator().manual_seed(5)
    theta0 = torch.randn(n_var, 32, 32, 4, dtype=torch.float64, generator=gen)

    def adam_loop(designs):
        """Warm-up and timed Adam steps from theta0; wall times, device times, objectives."""
        theta = theta0.clone().requires_grad_(True)
        opt = torch.optim.Adam([theta], lr=0.05)
        scale = None
        J_hist = []

        def adam_step():
            nonlocal scale
            opt.zero_grad()
            X = designs(list(1 + 9 * torch.sigmoid(theta)))
            J = (X.abs() ** 2).sum(dim=(1, 2))          # per variant
            if scale is None:
                scale = float(J.detach().mean())
            (-(J / scale).sum()).backward()               # maximise the output power of every variant
            opt.step()
            J_hist.append(J.detach().numpy() / scale)

        for _ in range(max(args.warmup, 1)):
            adam_step()
        t, fwd_ms, adj_ms = [], [], []
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            adam_step()
            torch.cuda.synchronize()
            t.append(time.perf_counter() - t0)
            st = designs.batch.stats()
            fwd_ms.append(st["last_run_ms"])
            adj_ms.append(st["adjoint_ms"])
        st = designs.batch.stats()
        designs.close()
        return theta.detach(), t, fwd_ms, adj_ms, st, J_hist

    th, t, fwd_ms, adj_ms, st, J_hist = adam_loop(FDTDDesignBatch([s] * n_var, box, terms, omega,
                                                                  checkpoint_every=every))
    _, t_rec, fwd_rec, adj_rec, _, _ = adam_loop(FDTDDesignBatch([s] * n_var, box, terms, omega,
                                                                 history_budget=float("inf")))
    # the same gradients one variant after another: one model, one forward
    # (same checkpoints) and one adjoint per variant
    single = FDTDDesign(s, box, terms, omega, checkpoint_every=every)

    def sequential_pass():
        for v in range(n_var):
            tv = th[v].clone().requires_grad_(True)
            (single(1 + 9 * torch.sigmoid(tv)).abs() ** 2).sum().backward()

    sequential_pass()  # warm-up
    t_seq = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sequential_pass()
        torch.cuda.synchronize()
        t_seq.append(time.perf_counter() - t0)
    single.close()
    ts = ranks.max(statistics.fmean(t))   # wall time of the slowest rank
    ts_rec = ranks.max(statistics.fmean(t_rec))
    ts_seq = ranks.max(statistics.fmean(t_seq))
    ranks.close()
    if rank != 0:
        return None
    cells = 96 * 96 * 64

    def device(fw, ad):
        return {"forward_ms": round(statistics.fmean(fw), 1), "adjoint_ms": round(statistics.fmean(ad), 1),
                "forward_mcell_updates_per_s": round(n_var * cells * nt / statistics.fmean(fw) / 1e3, 1),
                "adjoint_mcell_updates_per_s": round(n_var * cells * nt / statistics.fmean(ad) / 1e3, 1)}

    return {
        "metric": "grad evals/s", "value": round(world * n_var / ts, 3), "unit": "gradient evaluations/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ts * 1e3, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 fields, f64 accumulators",
        "data": "synthetic: microstrip background, seeded theta per variant",
        "config": {"workload": f"design: {n_var} variants of 96x96x64, 10-cell PML, {nt} steps, 32x32x4 design "
                               f"each, 5 freqs, Adam lr 0.05, checkpoints every {every}", "time_steps": nt,
                   "variants": n_var, "checkpoint_every": every,
                   "step": "one Adam step of all variants (batched forward with checkpoints + batched adjoint "
                           "with segment replays), wall time"},
        "device": device(fwd_ms, adj_ms),
        "objective_mean": [round(float(np.mean(j)), 4) for j in J_hist],
        "recorded_history": {"value": round(world * n_var / ts_rec, 3), "ms_per_step": round(ts_rec * 1e3, 1),
                             "device": device(fwd_rec, adj_rec),
                             "how": "the same Adam steps with every variant's box history recorded by the "
                                    "batched forward (no replay in the adjoint)"},
        "sequential": {"value": round(world * n_var / ts_seq, 3), "unit": "gradient evaluations/s",
                       "how": f"the {n_var} gradients one after another through FDTDDesign (forward with "
                              f"checkpoints every {every}, then the adjoint), wall time, no optimizer step"},
        "batched_over_sequential": round(ts_seq / ts, 3),
        "gpu_launches": int(st["step_launches"] + st["adjoint_launches"]),
    }


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        out = run_reference(args, rank, world)
    elif args.workload == "microstrip":
        out = run_microstrip(args, rank, world, local_rank)
    elif args.workload == "batch":
        out = run_batch(args, rank, world, local_rank)
    elif args.workload == "adjoint":
        out = run_adjoint(args, rank, world, local_rank)
    elif args.workload == "design":
        out = run_design(args, rank, world, local_rank)
    else:
        out, ctx = run_ours(args, rank, world, local_rank)
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline_entry()
        elif rank == 0:
            out["cpu_baseline"] = None
        if rank == 0 and world == 1 and not args.no_reference_cuda:
            out["reference_cuda"] = reference_cuda_entry(ctx)
        if rank == 0 and world == 1 and not args.no_workloads:
            out["workloads"] = workloads_entry(args, local_rank)
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
