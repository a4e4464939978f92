"""bench.py's host-side helpers on the CPU: the DRAM traffic and warp
instruction counts read from the committed ncu summaries, the stage bytes
behind each HBM fraction, the roofline peaks (measured file or the stated
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


def test_issue_roofline_reads_both_blend_captures():
    """The committed blend captures carry an instruction line each; the
    roofline is the pair arithmetic (scalar operations / 64) over the
    profiled warp instructions per contributing pair."""
    bw = {"fwd_pixel_pairs": 5, "bwd_pixel_pairs": 5}
    r = bench.issue_roofline(bw)
    for kernel, ops in (("blend_fwd", 17), ("blend_bwd", 29)):
        e = r[kernel]
        assert e["min_warp_inst_per_pair"] == round(ops / 64.0, 4)
        assert e["warp_inst_per_pair"] > e["min_warp_inst_per_pair"]
        assert 0.0 < e["frac"] < 1.0
        assert abs(e["frac"] - e["min_warp_inst_per_pair"] / e["warp_inst_per_pair"]) < 1e-3
    assert bench.profiled_instructions("no_such_stage") is None


def test_stage_bytes_follow_the_stated_formulas():
    """Algorithmic bytes per stage: the split-views step's last stage writes
    gradient rows only; BF16 storage halves the SH-rest and moment bytes."""
    N, V, P, K, items, tiles = 1000, 2, 64 * 48, 5000, 1200, 2 * 12
    bw = {"fwd_scanned": 900, "fwd_blended": 300, "bwd_scanned": 800, "bwd_blended": 250}
    full = bench.stage_bytes(N, V, P, K, items, bw, True, tiles)
    split = bench.stage_bytes(N, V, P, K, items, bw, True, tiles, adam=False)
    f32 = bench.stage_bytes(N, V, P, K, items, bw, False, tiles)
    assert full["project"] == N * (56 + 90) + V * N * 108
    assert full["depth_sort"] == V * N * 4 + 2 * V * N * 16
    assert full["item_sort"] == items * 20
    assert full["blend_fwd"] == 900 * 8 + 300 * 48 + V * P * 24
    assert full["blend_bwd"] == 800 * 8 + 250 * 48 + V * P * 36 + V * N * 48
    assert split["bwd_adam"] == V * N * 48 + N * 44 + N * 236 < full["bwd_adam"]
    assert f32["project"] - full["project"] == N * 90
    assert f32["bwd_adam"] > full["bwd_adam"]
    assert {k: v for k, v in split.items() if k != "bwd_adam"} == {k: v for k, v in full.items() if k != "bwd_adam"}
