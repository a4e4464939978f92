"""The autotuner's selection logic on the host: candidates, the coordinate
search over tile shape x binning path, then blend batch depth, then sort
digit width; rejected candidates skipped; deterministic ties.  A fake timer
stands in for the device steps (the device run is in tests/test_gpu_autotune.py)."""
import pytest

from nanotracer_b200._lib import SplatCudaError
from nanotracer_b200.autotune import (DIGIT_BITS, SORT_MODES, TILE_SHAPES, Trial, autotune, batch_choices,
                                      blend_threads, candidates, pick)
from nanotracer_b200.train import TrainConfig


def test_candidates_cover_every_tile_shape_and_binning_path():
    base = TrainConfig(n_views=3, width=640, height=480, bf16=True)
    cs = candidates(base)
    assert [(c.tile_w, c.tile_h, c.sort_mode) for c in cs] == \
        [(tw, th, sm) for (tw, th) in TILE_SHAPES for sm in SORT_MODES]
    # everything else is the base configuration
    assert all(c.n_views == 3 and c.width == 640 and c.bf16 for c in cs)


def test_batch_choices_are_whole_warps_within_the_blend_threads():
    assert blend_threads(16, 16) == 128 and blend_threads(8, 8) == 32 and blend_threads(32, 8) == 128
    assert batch_choices(16, 16) == [0, 64, 32]
    assert batch_choices(8, 8) == [0]
    assert batch_choices(32, 8) == [0, 64, 32]


def test_autotune_searches_each_axis_and_returns_the_fastest():
    times = {(16, 16, 0): 5.0, (16, 16, 1): 7.0, (8, 8, 0): 4.0, (8, 8, 1): 6.0, (32, 8, 1): 9.0,
             (32, 8, 0): 4.5}
    batch_bonus = {0: 0.0, 64: -0.5, 32: 0.3}
    digit_bonus = {0: 0.0, 8: 0.2, 9: -0.1}
    seen = []

    def timer(ctx, scene, cams, targets, cfg, warmup, steps):
        key = (cfg.tile_w, cfg.tile_h, cfg.sort_mode)
        seen.append((key, cfg.blend_batch, cfg.sort_digit_bits, warmup, steps))
        if key == (8, 8, 0):
            raise SplatCudaError(1, "tile rejected")  # status 1: invalid argument
        return times[key] + batch_bonus[cfg.blend_batch] + digit_bonus[cfg.sort_digit_bits], "same"

    base = TrainConfig(n_views=2, width=128, height=96, lrs=(1, 2, 3, 4, 5, 6), blend_batch=32, sort_digit_bits=8)
    best, trials = autotune(None, None, [], None, base, warmup=1, steps=4, timer=timer)
    # stage 1 (defaults for batch and digits): 32x8 two-level wins (8x8 rejected)
    assert all(s[1] == 0 and s[2] == 0 for s in seen[:6])
    assert (best.tile_w, best.tile_h, best.sort_mode) == (32, 8, 0)
    # stage 2: batch 64 wins; stage 3: 9-bit digits win
    assert best.blend_batch == 64 and best.sort_digit_bits == 9
    assert best.lrs == (1, 2, 3, 4, 5, 6) and best.n_views == 2
    assert len(trials) == len(TILE_SHAPES) * len(SORT_MODES) + 2 + len(DIGIT_BITS) == len(seen)
    assert all(w == 1 and s == 4 for *_, w, s in seen)
    failed = [t for t in trials if t.ms is None]
    assert [(t.tile_w, t.tile_h, t.sort_mode) for t in failed] == [(8, 8, 0)]
    assert "tile rejected" in failed[0].error


def test_pair_path_skips_the_batch_axis():
    def timer(ctx, scene, cams, targets, cfg, warmup, steps):
        return (1.0 if cfg.sort_mode == 1 else 2.0) + (0.1 if cfg.blend_batch else 0.0)

    best, trials = autotune(None, None, [], None, TrainConfig(), timer=timer)
    assert best.sort_mode == 1 and best.blend_batch == 0
    assert len(trials) == len(TILE_SHAPES) * len(SORT_MODES) + len(DIGIT_BITS)


def test_pick_prefers_the_earlier_of_equal_times_and_fails_when_nothing_ran():
    t = [Trial(16, 16, 0, 3.0, None), Trial(8, 8, 0, 3.0, None), Trial(32, 8, 0, None, "x")]
    assert pick(t) == 0
    with pytest.raises(RuntimeError, match="no candidate"):
        pick([Trial(16, 16, 0, None, "oom")])
