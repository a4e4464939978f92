"""Autotuner for the batched training step.

The reference has no tuner: its tile size is a fixed argument
(TilingParams, crates/nano-optimize/src/tile_binner.rs:21-42), its blend
stages one splat per workgroup thread, and its sort is a fixed 32-pass 1-bit
split (radix_sort.rs:1-26).  Here the choices that change the step's speed
but not what it computes are picked by timing: each candidate configuration
runs a few steps on a scratch copy of the scene, and the fastest is returned.

Tuned axes:
  * tile shape: 16x16, 8x8, 32x8;
  * binning path: two-level super-tile item lists, or the stable sort of the
    (tile, splat) pairs (TrainConfig.sort_mode);
  * blend batch depth: list positions the blend kernels stage per batch
    (TrainConfig.blend_batch: a quarter, half or all of the tile's threads);
  * sort radix width: 8- or 9-bit digits in the binning sort's onesweep
    passes (TrainConfig.sort_digit_bits).
The search is coordinate-wise: tile shape x binning path first (with the
default batch and digits), then the batch depth on the best of those, then
the digit width on the best batch; 11 trials at most instead of 36.

The binning path, the batch depth and the digit width never change the
images: every pixel blends the same splats in the same order.  The tile shape
can, as in the reference: a splat is listed in the tiles of its 3-sigma
rectangle rounded out to whole tiles, and the blend evaluates every pixel of a
listed tile, so a pixel just beyond 3 sigma (where alpha still passes 1/255
for opacities near 1) takes the splat in some tilings and not in others (on
1M splats at 1080p about 1 % of the pixels, by at most 0.015).  Tuning the
tile shape is choosing the reference's tile_size, a training parameter there;
pass tiles=[(tile_w, tile_h)] to keep the caller's.  The device test checks
that candidates with the same tile shape render bit-identical first steps.

The scratch copies mean that tuning leaves the caller's splats, moments and
trainer untouched; it costs one upload and one trainer per candidate.
"""
from __future__ import annotations

import gc
import hashlib
import time
from dataclasses import dataclass, replace
from typing import Callable, Optional

from ._lib import SplatCudaError
from .gpu import CudaCtx, DeviceBuffer
from .raster import CameraUniform
from .splat_gpu import AdamMomentBuffers, GpuSplatBuffer
from .splat_store import SplatBuffer
from .train import TrainConfig, Trainer

TILE_SHAPES = ((16, 16), (8, 8), (32, 8))
SORT_MODES = (0, 1)        # TrainConfig.sort_mode: two-level item lists, stable pair sort
BATCH_FRACTIONS = (4, 2)   # blend batch = threads / f, besides the default (all threads)
DIGIT_BITS = (8, 9)        # TrainConfig.sort_digit_bits, besides the default (fewer passes wins)


@dataclass
class Trial:
    tile_w: int
    tile_h: int
    sort_mode: int
    ms: Optional[float]    # mean step time, None when the candidate failed
    error: Optional[str]   # the library's message for a failed candidate
    blend_batch: int = 0
    sort_digit_bits: int = 0
    digest: Optional[str] = None  # hash of the first step's images

    @property
    def label(self) -> str:
        return (f"{self.tile_w}x{self.tile_h}/sort_mode {self.sort_mode}/batch {self.blend_batch or 'all'}"
                f"/digits {self.sort_digit_bits or 'auto'}")


def blend_threads(tile_w: int, tile_h: int) -> int:
    """Threads of a blend CTA: two pixels per thread when the tile splits into
    whole warps that way, else one (k_blend.cu pick_ppt)."""
    px = tile_w * tile_h
    return px // 2 if (tile_h % 2 == 0 and (px // 2) % 32 == 0) else px


def batch_choices(tile_w: int, tile_h: int) -> list[int]:
    """Blend batch depths worth trying for a tile shape (0 = all threads)."""
    th = blend_threads(tile_w, tile_h)
    return [0] + sorted({th // f for f in BATCH_FRACTIONS if th // f >= 32 and (th // f) % 32 == 0}, reverse=True)


def candidates(base: TrainConfig, tiles=TILE_SHAPES, sort_modes=SORT_MODES) -> list[TrainConfig]:
    """First stage of the search: base with each tile shape and binning path."""
    return [replace(base, tile_w=tw, tile_h=th, sort_mode=sm) for (tw, th) in tiles for sm in sort_modes]


def pick(trials: list[Trial]) -> int:
    """Index of the fastest trial that ran; the earlier one wins a tie, so the
    choice is deterministic for equal timings."""
    best = None
    for i, t in enumerate(trials):
        if t.ms is not None and (best is None or t.ms < trials[best].ms):
            best = i
    if best is None:
        raise RuntimeError("autotune: no candidate configuration ran: " +
                           "; ".join(f"{t.label}: {t.error}" for t in trials))
    return best


def time_steps(ctx: CudaCtx, scene: SplatBuffer, cams: list[CameraUniform], targets: DeviceBuffer,
               cfg: TrainConfig, warmup: int = 2, steps: int = 3):
    """(mean wall time in ms of `steps` training steps of `cfg` on a fresh
    device copy of `scene` after `warmup` untimed steps, hash of the first
    step's images).  The first warm-up step captures the step's graph; each
    step reads its loss back, so the host clock brackets finished device work."""
    g = GpuSplatBuffer.upload(ctx, scene, bf16_rest=cfg.bf16)
    mo = AdamMomentBuffers(ctx, g.capacity, bf16=cfg.bf16)
    acc = ctx.storage_buffer_zeroed("autotune_acc", 4 * g.capacity)
    tr = Trainer(ctx, cfg)
    try:
        tr.set_targets(targets)
        t = 1
        tr.step(g, mo, acc, cams, t)
        digest = hashlib.sha256(tr.images().tobytes()).hexdigest()
        for _ in range(max(0, warmup - 1)):
            t += 1
            tr.step(g, mo, acc, cams, t)
        t0 = time.perf_counter()
        for _ in range(steps):
            t += 1
            tr.step(g, mo, acc, cams, t)
        return (time.perf_counter() - t0) * 1e3 / steps, digest
    finally:
        del tr, acc, mo, g
        gc.collect()


def _run(timer, ctx, scene, cams, targets, cfg, warmup, steps) -> Trial:
    try:
        r = timer(ctx, scene, cams, targets, cfg, warmup, steps)
        ms, digest = r if isinstance(r, tuple) else (r, None)
        return Trial(cfg.tile_w, cfg.tile_h, cfg.sort_mode, float(ms), None, cfg.blend_batch, cfg.sort_digit_bits,
                     digest)
    except SplatCudaError as e:
        return Trial(cfg.tile_w, cfg.tile_h, cfg.sort_mode, None, str(e), cfg.blend_batch, cfg.sort_digit_bits)


def autotune(ctx: CudaCtx, scene: SplatBuffer, cams: list[CameraUniform], targets: DeviceBuffer,
             base: TrainConfig, tiles=TILE_SHAPES, sort_modes=SORT_MODES, warmup: int = 2, steps: int = 3,
             timer: Callable = time_steps, tune_batch: bool = True,
             tune_digits: bool = True) -> tuple[TrainConfig, list[Trial]]:
    """Time the candidates on `scene` with `cams` and the device `targets`
    (float3 per pixel, as Trainer.set_targets takes) and return `base` with
    the fastest tile shape, binning path, blend batch depth and sort digit
    width, plus every trial.  A candidate the library rejects (a tile shape
    that does not fit its blend kernel, an allocation that fails) is recorded
    with its error and skipped; if none runs, RuntimeError."""
    trials = [_run(timer, ctx, scene, cams, targets, cfg, warmup, steps)
              for cfg in candidates(replace(base, blend_batch=0, sort_digit_bits=0), tiles, sort_modes)]
    b = trials[pick(trials)]
    best = replace(base, tile_w=b.tile_w, tile_h=b.tile_h, sort_mode=b.sort_mode, blend_batch=0, sort_digit_bits=0)
    best_trial = b
    if tune_batch and best.sort_mode != 1:  # the batch depth applies to the item-list blends
        stage = [best_trial] + [_run(timer, ctx, scene, cams, targets, replace(best, blend_batch=bb), warmup, steps)
                                for bb in batch_choices(best.tile_w, best.tile_h) if bb != 0]
        trials += stage[1:]
        best_trial = stage[pick(stage)]
        best = replace(best, blend_batch=best_trial.blend_batch)
    if tune_digits:
        stage = [best_trial] + [_run(timer, ctx, scene, cams, targets, replace(best, sort_digit_bits=d), warmup,
                                     steps) for d in DIGIT_BITS]
        trials += stage[1:]
        best_trial = stage[pick(stage)]
        best = replace(best, sort_digit_bits=best_trial.sort_digit_bits)
    return best, trials
