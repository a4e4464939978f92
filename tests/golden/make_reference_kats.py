"""Writes tests/golden/reference_kats.json: the known-answer vectors and
tolerances of the reference's own test suite for this path, transcribed from
its Rust test sources (ssoj13/nanotracer; paths relative to the project root).
The reference keeps no golden files on disk — every fixture there is built in
code — so this file records those inputs and expected outputs as data.

    python tests/golden/make_reference_kats.py
"""
import json
import math
from pathlib import Path

KATS = {
    "cpu_oracle_centers_on_axis": {
        "source": "crates/nano-optimize/src/raster.rs:999-1026 (unit_splat :974-986, standard_camera :988-997)",
        "splat": {"pos": [0.0, 0.0, -5.0], "rot": [1.0, 0.0, 0.0, 0.0], "log_scale": [0.0, 0.0, 0.0],
                  "opacity_logit": 10.0, "sh_dc": [0.5, 0.3, 0.1]},
        "camera": {"eye": [0.0, 0.0, 0.0], "target": [0.0, 0.0, -1.0], "up": [0.0, 1.0, 0.0],
                   "fov_y": math.pi / 2, "width": 256, "height": 256},
        "expect": {"visible": 1.0, "mean": [128.0, 128.0], "mean_tol": 1e-3, "depth": 5.0, "depth_tol": 1e-3,
                   "radius_open_interval": [50.0, 100.0], "conic_b_abs_max": 1e-3, "conic_a_minus_c_abs_max": 1e-3},
    },
    "wgsl_matches_cpu_oracle_tolerances": {
        "source": "crates/nano-optimize/src/raster.rs:1217-1265",
        "tol": {"mean": 1e-2, "depth": 1e-3, "radius": 1.0, "conic": 1e-4, "color": 1e-3, "opacity": 1e-5},
    },
    "composite_single_splat_renders_gaussian": {
        "source": "crates/nano-optimize/src/raster.rs:1028-1100",
        "record": {"mean_xy": [32.5, 32.5], "depth": 5.0, "radius": 30.0, "conic": [0.04, 0.0, 0.04],
                   "visible": 1.0, "color": [1.0, 1.0, 1.0], "opacity": 1.0},
        "tiling": {"width": 64, "height": 64, "tile_size": 16, "depth_max": 100.0},
        "expect": {"centre_xy": [32, 32], "centre_rgb_min": 0.9, "centre_alpha_min": 0.9, "near_xy": [34, 34],
                   "near_rgb_min": 0.6, "edge_xy": [0, 0], "edge_rgb_max": 0.05, "edge_alpha_max": 0.05,
                   "diag_steps": 16, "diag_tol": 1e-3},
    },
    "backward_accumulates_per_splat_gradients": {
        "source": "crates/nano-optimize/src/raster.rs:1102-1215",
        "record": {"mean_xy": [16.0, 16.0], "depth": 5.0, "radius": 25.0, "conic": [0.04, 0.0, 0.04],
                   "visible": 1.0, "color": [1.0, 1.0, 1.0], "opacity": 1.0},
        "tiling": {"width": 32, "height": 32, "tile_size": 16, "depth_max": 100.0},
        "dl_dc": [1.0, 1.0, 1.0, 0.0],
        "expect": {"dcolor_min": 0.1, "dopacity_min": 0.01, "dconic_a_max": -1e-4, "dconic_c_max": -1e-4,
                   "dmean_abs_max": 0.5},
    },
    "four_splats_bin_to_expected_tiles": {
        "source": "crates/nano-optimize/src/tile_binner.rs:443-501",
        "records": [[8.0, 8.0, 10.0, 4.0], [40.0, 8.0, 20.0, 4.0], [8.0, 56.0, 30.0, 4.0], [56.0, 56.0, 5.0, 4.0]],
        "record_fields": "mean_x, mean_y, depth, radius; conic (1,0,1), visible 1, colour 1, opacity 1",
        "tiling": {"width": 64, "height": 64, "tile_size": 16, "depth_max": 100.0},
        "expect": {"total_pairs": 4, "num_tiles": 16, "tiles": [0, 2, 12, 15],
                   "ranges": [[0, 0, 1], [2, 1, 2], [12, 2, 3], [15, 3, 4]], "payloads": [0, 1, 2, 3]},
    },
    "two_splats_same_tile_sorted_by_depth": {
        "source": "crates/nano-optimize/src/tile_binner.rs:503-541",
        "records": [[24.0, 24.0, 80.0, 4.0], [24.0, 24.0, 5.0, 4.0]],
        "tiling": {"width": 64, "height": 64, "tile_size": 16, "depth_max": 100.0},
        "expect": {"total_pairs": 2, "tiles": [5, 5], "payloads": [1, 0], "tile5_range": [0, 2]},
    },
    "sort_small_array_stable": {
        "source": "crates/nano-optimize/src/radix_sort.rs:357-379",
        "keys": [3, 1, 4, 1, 5, 9, 2, 6], "vals": [0, 1, 2, 3, 4, 5, 6, 7],
        "expect": {"keys": [1, 1, 2, 3, 4, 5, 6, 9], "vals_prefix": [1, 3]},
    },
    "sort_random_u32_with_payload": {
        "source": "crates/nano-optimize/src/radix_sort.rs:381-408",
        "n": 10000, "lcg": {"seed": 0xDEADBEEF, "a": 1664525, "c": 1013904223, "key": "state after each step"},
    },
    "scan_all_ones_yields_indices": {"source": "crates/nano-optimize/src/prefix_scan.rs:305-319", "n": 1000},
    "scan_random_matches_cpu_reference": {
        "source": "crates/nano-optimize/src/prefix_scan.rs:321-333",
        "n": 70000, "lcg": {"seed": 0x12345678, "a": 1664525, "c": 1013904223, "value": "state % 17"},
    },
    "roundtrip_upload_readback": {"source": "crates/nano-optimize/src/splat_gpu.rs:451-473", "bit_exact": True},
    "swap_remove_keeps_invariants": {
        "source": "crates/nano-optimize/src/splat_store.rs:157-176",
        "n": 5, "remove": 1, "expect": {"len": 4, "sh_rest_len": 180, "positions_1": [4.0, 4.0, 4.0]},
    },
    "adam_basics": {
        "source": "crates/nano-optimize/src/adam.rs:119-149",
        "defaults": {"lr": 1.6e-4, "beta1": 0.9, "beta2": 0.999, "eps": 1e-15},
    },
    "adam_gpu_parity": {
        "source": "crates/nano-optimize/tests/adam_gpu_parity.rs:20-412",
        "param_tol": 1e-4, "moment_tol": 1e-5, "init_param": 0.5,
        "runs": [
            {"n": 256, "steps": 10, "grad": "0.1"},
            {"n": 256, "steps": 10, "grad": "-0.2"},
            {"n": 1024, "steps": 20, "grad": "(1 if i%2==0 else -1) * (0.05 + 0.01*t)"},
            {"n": 64, "steps": 1, "grad": "0.01*(i+1)"},
            {"n": 8192, "steps": 5, "grad": "0.05*sin(0.01*i + 0.1*t)"},
        ],
        "step_all_pos_lr": 5e-4,
    },
    "densify_clones_small_and_splits_large": {
        "source": "crates/nano-optimize/src/train.rs:626-697",
        "splats": [
            {"pos": [0.0, 0.0, 0.0], "rot": [1.0, 0.0, 0.0, 0.0], "scale": [-3.0, -3.0, -3.0], "opacity": 2.0,
             "dc": [0.5, 0.5, 0.5]},
            {"pos": [5.0, 5.0, 5.0], "rot": [1.0, 0.0, 0.0, 0.0], "scale": [0.0, 0.0, 0.0], "opacity": 2.0,
             "dc": [0.3, 0.3, 0.3]},
            {"pos": [-1.0, -1.0, -1.0], "rot": [1.0, 0.0, 0.0, 0.0], "scale": [-1.0, -1.0, -1.0], "opacity": 2.0,
             "dc": [0.1, 0.2, 0.3]},
        ],
        "grad_acc": [1.0, 1.0, 0.0001], "grad_count": 1, "threshold": 0.5, "split_thr": -2.3, "max_splats": 100,
        "iter": 42,
        "expect": {"cloned": 1, "split_children": 2, "removed": 1, "len": 5},
    },
    "prune_drops_low_opacity_splats": {
        "source": "crates/nano-optimize/src/train.rs:699-743",
        "opacities": [2.0, -10.0, 2.0, -10.0, 2.0], "grad_acc": [10.0, 20.0, 30.0, 40.0, 50.0], "threshold": -5.3,
        "expect": {"removed": 2, "len": 3, "survivor_opacity": 2.0},
    },
    "finite_diff_matches_analytic": {
        "source": "crates/nano-optimize/tests/backward_finite_diff.rs:28-246",
        "splat": {"pos": [0.0, 0.0, -5.0], "rot": [1.0, 0.0, 0.0, 0.0], "log_scale": [-0.5, -0.6, -0.7],
                  "opacity_logit": 2.0, "sh_dc": [0.4, 0.3, 0.2], "sh_rest": {"0": 0.05, "20": -0.03}},
        "camera": {"eye": [0.0, 0.0, 0.0], "target": [0.0, 0.0, -1.0], "up": [0.0, 1.0, 0.0], "fov_y": math.pi / 3,
                   "width": 32, "height": 32},
        "tiling": {"tile_size": 16, "depth_max": 50.0},
        "loss": "sum of rgb over all pixels", "eps": 1e-3,
        "checks": {"sh_dc.r": [0.02, 0.05], "opacity": [0.05, 0.05], "sh_rest[0]": [0.05, 0.05],
                   "pos.x": [0.10, 0.5], "log_scale.x": [0.10, 0.5]},
        "close": "|a-n| <= abs or |a-n| <= rel*(|a|+|n|)",
    },
    "ply_write_then_read_roundtrip": {
        "source": "crates/nano-splat/src/ply.rs:262-287",
        "gaussian": {"pos": [1.0, 2.0, 3.0], "normal": [0.0, 1.0, 0.0], "sh_dc": [0.4, 0.5, 0.6],
                     "sh_rest": "i*0.1 for i in 0..45", "opacity": 2.7, "scale": [-0.5, -0.6, -0.7],
                     "rotation": [1.0, 0.0, 0.0, 0.0]},
        "rest_tol": 1e-5,
    },
}

if __name__ == "__main__":
    out = Path(__file__).with_name("reference_kats.json")
    out.write_text(json.dumps(KATS, indent=1, sort_keys=True) + "\n")
    print(f"wrote {out}")
