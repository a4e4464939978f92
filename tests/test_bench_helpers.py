"""bench.py's host-side helpers on the CPU: the DRAM traffic read from the
committed ncu summaries, the roofline peaks (measured file or the stated
fallback) and the clock-sample summary that accepts or rejects a run."""
import json
import time

import bench


def test_profiled_traffic_scales_the_capture_by_views():
    two = bench.profiled_traffic("blend_bwd", 2)
    assert two is not None and two > 0
    assert bench.profiled_traffic("blend_bwd", 8) == 4 * two
    assert bench.profiled_traffic("no_such_stage", 8) is None


def test_peaks_come_from_the_measured_file_else_the_fallback(tmp_path, monkeypatch):
    monkeypatch.setattr(bench, "ROOT", tmp_path)
    assert bench.load_peaks() == {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}
    (tmp_path / "MEASURED_PEAKS.json").write_text(json.dumps({"hbm_gbs": 6452.5, "bf16_tflops": 1601.0}))
    assert bench.load_peaks() == {"hbm_gbs": 6452.5, "bf16_tflops": 1601.0, "source": "measured"}


def _sample(ts, sm, reasons):
    # nvidia-smi --format=csv,noheader,nounits with the sampler's query columns
    stamp = time.strftime("%Y/%m/%d %H:%M:%S", time.localtime(ts)) + f".{int((ts % 1) * 1000):03d}"
    flags = ["Active" if r else "Not Active" for r in reasons]
    return ", ".join([stamp, "0", str(sm), "1965", "700.0", "0x0"] + flags)


def test_clock_summary_keeps_the_timed_window_and_names_active_reasons(tmp_path):
    s = bench.ClockSampler(0)
    t0 = time.time()
    rows = [_sample(t0 - 5.0, 1200, (True, False, False, False)),   # before the window: ignored
            _sample(t0 + 0.1, 1965, (False, False, False, True)),
            _sample(t0 + 0.2, 1950, (False, False, False, False)),
            _sample(t0 + 0.3, 1965, (False, False, False, False))]
    s.path.write_text("\n".join(rows) + "\n")
    got = s.summary(t0, t0 + 0.35)
    assert got == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": ["sw_power_cap"], "samples": 3}
    s.path.write_text("")
    assert s.summary(t0, t0 + 1)["reasons"] == ["unsampled"]
