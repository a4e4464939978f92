"""The autotuner on the device: every candidate (tile shape x binning path)
runs and is timed, the returned configuration is the fastest one, and a
trainer built from it steps the scene."""
import math

import numpy as np
import pytest

from nanotracer_b200 import AdamMomentBuffers, CameraUniform, GpuSplatBuffer, TilingParams
from nanotracer_b200.autotune import SORT_MODES, TILE_SHAPES, autotune
from nanotracer_b200.scene import FOV_Y, orbit_views, perturbed, random_scene
from nanotracer_b200.train import TrainConfig, Trainer, render_targets

pytestmark = pytest.mark.gpu


def test_autotune_times_every_candidate_and_returns_the_fastest(ctx):
    n, W, H, V = 4000, 160, 128, 2
    scene = random_scene(n, 33)
    tl = TilingParams(W, H, 16, 8.0, tile_h_override=16)
    cams = [CameraUniform.from_pose(*p, FOV_Y, W, H, n) for p in orbit_views(V, 0)]
    tbuf = ctx.storage_buffer("targets", np.ascontiguousarray(render_targets(ctx, perturbed(scene), cams, tl),
                                                               np.float32))
    base = TrainConfig(n_views=V, width=W, height=H, depth_max=8.0, exact_backward=True, use_graph=True)
    best, trials = autotune(ctx, scene, cams, tbuf, base, warmup=1, steps=2)
    assert len(trials) == len(TILE_SHAPES) * len(SORT_MODES)
    assert all(t.error is None and t.ms > 0 for t in trials)
    fastest = min(trials, key=lambda t: t.ms)
    assert (best.tile_w, best.tile_h, best.sort_mode) == (fastest.tile_w, fastest.tile_h, fastest.sort_mode)
    # the chosen configuration trains the caller's own copy of the scene
    g = GpuSplatBuffer.upload(ctx, scene)
    mo = AdamMomentBuffers(ctx, g.capacity)
    acc = ctx.storage_buffer_zeroed("acc", 4 * g.capacity)
    tr = Trainer(ctx, best)
    tr.set_targets(tbuf)
    losses = [tr.step(g, mo, acc, cams, t) for t in (1, 2)]
    assert all(math.isfinite(x) and x > 0 for x in losses)
