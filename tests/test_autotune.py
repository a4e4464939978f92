"""The autotuner's selection logic on the host: candidates, the fastest pick,
rejected candidates skipped, deterministic ties.  A fake timer stands in for
the device steps (the device run is in tests/test_gpu_autotune.py)."""
import pytest

from nanotracer_b200._lib import SplatCudaError
from nanotracer_b200.autotune import SORT_MODES, TILE_SHAPES, Trial, autotune, candidates, pick
from nanotracer_b200.train import TrainConfig


def test_candidates_cover_every_tile_shape_and_binning_path():
    base = TrainConfig(n_views=3, width=640, height=480, bf16=True)
    cs = candidates(base)
    assert [(c.tile_w, c.tile_h, c.sort_mode) for c in cs] == \
        [(tw, th, sm) for (tw, th) in TILE_SHAPES for sm in SORT_MODES]
    # everything else is the base configuration
    assert all(c.n_views == 3 and c.width == 640 and c.bf16 for c in cs)


def test_autotune_returns_the_fastest_and_skips_rejected_candidates():
    times = {(16, 16, 0): 5.0, (16, 16, 1): 7.0, (8, 8, 0): 4.0, (8, 8, 1): 6.0, (32, 8, 1): 9.0}
    seen = []

    def timer(ctx, scene, cams, targets, cfg, warmup, steps):
        key = (cfg.tile_w, cfg.tile_h, cfg.sort_mode)
        seen.append((key, warmup, steps))
        if key not in times:
            raise SplatCudaError(1, "tile rejected")  # status 1: invalid argument
        return times[key]

    base = TrainConfig(n_views=2, width=128, height=96, lrs=(1, 2, 3, 4, 5, 6))
    best, trials = autotune(None, None, [], None, base, warmup=1, steps=4, timer=timer)
    assert (best.tile_w, best.tile_h, best.sort_mode) == (8, 8, 0)
    assert best.lrs == (1, 2, 3, 4, 5, 6) and best.n_views == 2
    assert len(trials) == len(TILE_SHAPES) * len(SORT_MODES) == len(seen)
    assert all(w == 1 and s == 4 for _, w, s in seen)
    failed = [t for t in trials if t.ms is None]
    assert [(t.tile_w, t.tile_h, t.sort_mode) for t in failed] == [(32, 8, 0)]
    assert "tile rejected" in failed[0].error


def test_pick_prefers_the_earlier_of_equal_times_and_fails_when_nothing_ran():
    t = [Trial(16, 16, 0, 3.0, None), Trial(8, 8, 0, 3.0, None), Trial(32, 8, 0, None, "x")]
    assert pick(t) == 0
    with pytest.raises(RuntimeError, match="no candidate"):
        pick([Trial(16, 16, 0, None, "oom")])
