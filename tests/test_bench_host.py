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
