"""bench.py's host-side helpers on the CPU: the roofline peak (measured file or
the fallback), the profiled DRAM traffic read from the committed ncu summary,
and the clock sampler's summary of nvidia-smi samples (median SM clock, the
throttle reasons seen)."""
import json

import bench


def test_peak_fallback_and_measured(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench.peaks() == (bench.FALLBACK_HBM_GBS, "fallback")
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6549.4, "bf16_tflops": 1590.0}))
    assert bench.peaks() == (6549.4, "measured")


def test_profiled_traffic_of_the_committed_summary(tmp_path):
    assert bench.profiled_traffic(1) == 636571136          # profiles/fdtd_step_stream_boxes256.md
    assert bench.profiled_traffic(0) is None               # the plain kernel's is not recorded there
    assert bench.profiled_traffic(1, tmp_path / "missing.md") is None


def test_clock_summary(tmp_path):
    c = bench.ClockSampler(0)
    c.path = tmp_path / "clocks.csv"
    c.proc = object()   # as if nvidia-smi had run
    rows = ["0, 1965, 1965, 700.1, 0x0, Not Active, Not Active, Not Active, Not Active",
            "0, 1905, 1965, 995.2, 0x4, Not Active, Not Active, Not Active, Active",
            "0, 1935, 1965, 990.0, 0x4, Not Active, Not Active, Not Active, Active",
            "garbage"]
    c.path.write_text("\n".join(rows) + "\n")
    out = c.summary()
    assert out["sm_mhz"] == 1935.0 and out["sm_max_mhz"] == 1965.0
    assert out["reasons"] == ["sw_power_cap"] and out["samples"] == 3


def test_reference_arm_line_matches_our_contract(monkeypatch):
    """`bench.py --impl reference` (the CPU restatement of the reference
    engine, on a bounded sample) prints the metric, unit, direction and config
    of this engine's line, with zero host-device bytes."""
    import argparse

    from oracle import cpu_engine
    monkeypatch.setattr(bench, "sample_steps", lambda n_threads, seconds=10.0: 2)
    monkeypatch.setattr(cpu_engine, "default_threads", lambda: 2)
    args = argparse.Namespace(steps=1, warmup=0, nt=bench.NT)
    line = bench.run_reference(args, 0, 1)
    assert bench.run_reference(args, 1, 2) is None          # other ranks print nothing
    assert line["impl"] == "reference"
    assert (line["metric"], line["unit"], line["higher_is_better"]) == (bench.METRIC, bench.UNIT, True)
    s = bench.build_model(2)
    co, pr, *_ = s.pack_inputs(gpu=True)
    names, _, _ = bench.dft_spec(s, pr)
    assert line["config"] == bench.bench_config(bench.NT, 1, len(names), len(pr))
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["e2e"]["value"] == line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] == 2
    json.dumps(line)


def test_cpu_baseline_entry_reports_host_and_default_threads(monkeypatch):
    from oracle import cpu_engine
    monkeypatch.setattr(bench, "sample_steps", lambda n_threads, seconds=10.0: 2)
    monkeypatch.setattr(cpu_engine, "default_threads", lambda: 2)
    calls = []
    real = bench.cpu_sample
    monkeypatch.setattr(bench, "cpu_sample", lambda nt, n: calls.append((nt, n)) or real(2, n))
    out = bench.cpu_baseline_entry()
    assert calls == [(2, 2), (8, 4)]
    assert out["kind"] == "port" and out["cores"] == 2 and out["value"] > 0
    assert out["host"]["nproc"] >= 1 and isinstance(out["host"]["cpu"], str)
    assert out["at_reference_default_threads"]["cores"] == 4 and out["at_reference_default_threads"]["value"] > 0
    json.dumps(out)
