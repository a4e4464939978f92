"""The autotuner on the device: every candidate of its coordinate search
(tile shape x binning path, blend batch depth, sort digit width) runs and is
timed, candidates with the same tile shape render bit-identical first steps
(the binning path, batch depth and digit width change speed, not results; the
tile shape decides, as the reference's tile_size does, which pixels just past
a splat's 3-sigma rectangle see it), the returned configuration is each
stage's fastest, and a trainer built from it steps the scene."""
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
    assert len(trials) >= len(TILE_SHAPES) * len(SORT_MODES) + 2
    assert all(t.error is None and t.ms > 0 for t in trials), [t.label for t in trials if t.error]
    for shape in {(t.tile_w, t.tile_h) for t in trials}:
        same = [t for t in trials if (t.tile_w, t.tile_h) == shape]
        assert len({t.digest for t in same}) == 1, [(t.label, t.digest[:8]) for t in same]
    stage1 = trials[:len(TILE_SHAPES) * len(SORT_MODES)]
    f1 = min(stage1, key=lambda t: t.ms)
    assert (best.tile_w, best.tile_h, best.sort_mode) == (f1.tile_w, f1.tile_h, f1.sort_mode)
    chosen = [t for t in trials if (t.tile_w, t.tile_h, t.sort_mode, t.blend_batch, t.sort_digit_bits) ==
              (best.tile_w, best.tile_h, best.sort_mode, best.blend_batch, best.sort_digit_bits)]
    assert chosen
    print({t.label: round(t.ms, 3) for t in trials})
    # the chosen configuration trains the caller's own copy of the scene
    g = GpuSplatBuffer.upload(ctx, scene)
    mo = AdamMomentBuffers(ctx, g.capacity)
    acc = ctx.storage_buffer_zeroed("acc", 4 * g.capacity)
    tr = Trainer(ctx, best)
    tr.set_targets(tbuf)
    losses = [tr.step(g, mo, acc, cams, t) for t in (1, 2)]
    assert all(math.isfinite(x) and x > 0 for x in losses)


@pytest.mark.parametrize("batch", [32, 64])
@pytest.mark.parametrize("digits", [8, 9])
def test_blend_batch_and_digit_width_leave_the_step_unchanged(ctx, batch, digits):
    """A non-default blend batch depth and sort digit width give the default
    configuration's forward bit for bit and its first Adam step except where
    a gradient's sign is within the float atomics' ordering noise
    (tests/util.py check_same_first_step)."""
    from tests.util import check_same_first_step
    n, W, H, V = 6000, 256, 192, 2
    scene = random_scene(n, 44)
    tl = TilingParams(W, H, 16, 8.0)
    cams = [CameraUniform.from_pose(*p, FOV_Y, W, H, n) for p in orbit_views(V, 0)]
    tgt = render_targets(ctx, perturbed(scene), cams, tl)
    out = []
    for cfg in (TrainConfig(n_views=V, width=W, height=H, depth_max=8.0),
                TrainConfig(n_views=V, width=W, height=H, depth_max=8.0, blend_batch=batch, sort_digit_bits=digits)):
        g = GpuSplatBuffer.upload(ctx, scene)
        mo = AdamMomentBuffers(ctx, g.capacity)
        acc = ctx.storage_buffer_zeroed("acc", 4 * g.capacity)
        tr = Trainer(ctx, cfg)
        tr.set_targets(ctx.storage_buffer("t", np.ascontiguousarray(tgt, np.float32)))
        loss = tr.step(g, mo, acc, cams, 1)
        out.append((tr.images(), loss, g.readback().flat()))
    assert np.array_equal(out[0][0], out[1][0])
    assert abs(out[0][1] - out[1][1]) <= 1e-12 * out[0][1]
    print(check_same_first_step(out[0][2], out[1][2], cfg.lrs))
