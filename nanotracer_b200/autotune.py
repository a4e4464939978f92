"""Autotuner for the batched training step.

The reference has no tuner: its tile size is a fixed argument
(TilingParams, crates/nano-optimize/src/tile_binner.rs) and its sort a fixed
32-pass split.  Here the choices that change the step's speed but not what it
computes are picked by timing: each candidate configuration runs a few steps
on a scratch copy of the scene, and the fastest is returned.

Tuned: the tile shape (8x8, 16x16, 32x8) and the binning path (two-level
super-tile item lists, or the stable sort of the (tile, splat) pairs).  The
blend batch depth follows from the tile (one CTA per tile, a batch of one
list position per thread, two pixels per thread), and the sort's digit width
is chosen inside the sort from the key width, so neither is a separate axis.

The scratch copies mean that tuning leaves the caller's splats, moments and
trainer untouched; it costs one upload and one trainer per candidate.
"""
from __future__ import annotations

import gc
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
SORT_MODES = (0, 1)  # TrainConfig.sort_mode: two-level item lists, stable pair sort


@dataclass
class Trial:
    tile_w: int
    tile_h: int
    sort_mode: int
    ms: Optional[float]    # mean step time, None when the candidate failed
    error: Optional[str]   # the library's message for a failed candidate


def candidates(base: TrainConfig, tiles=TILE_SHAPES, sort_modes=SORT_MODES) -> list[TrainConfig]:
    """The configurations tried: base with each tile shape and binning path."""
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
                           "; ".join(f"{t.tile_w}x{t.tile_h}/{t.sort_mode}: {t.error}" for t in trials))
    return best


def time_steps(ctx: CudaCtx, scene: SplatBuffer, cams: list[CameraUniform], targets: DeviceBuffer,
               cfg: TrainConfig, warmup: int = 2, steps: int = 3) -> float:
    """Mean wall time in ms of `steps` training steps of `cfg` on a fresh
    device copy of `scene`, after `warmup` untimed steps (the first one
    captures the step's graph).  Each step reads its loss back, so the host
    clock brackets finished device work."""
    g = GpuSplatBuffer.upload(ctx, scene, bf16_rest=cfg.bf16)
    mo = AdamMomentBuffers(ctx, g.capacity, bf16=cfg.bf16)
    acc = ctx.storage_buffer_zeroed("autotune_acc", 4 * g.capacity)
    tr = Trainer(ctx, cfg)
    try:
        tr.set_targets(targets)
        t = 0
        for _ in range(warmup):
            t += 1
            tr.step(g, mo, acc, cams, t)
        t0 = time.perf_counter()
        for _ in range(steps):
            t += 1
            tr.step(g, mo, acc, cams, t)
        return (time.perf_counter() - t0) * 1e3 / steps
    finally:
        del tr, acc, mo, g
        gc.collect()


def autotune(ctx: CudaCtx, scene: SplatBuffer, cams: list[CameraUniform], targets: DeviceBuffer,
             base: TrainConfig, tiles=TILE_SHAPES, sort_modes=SORT_MODES, warmup: int = 2, steps: int = 3,
             timer: Callable[..., float] = time_steps) -> tuple[TrainConfig, list[Trial]]:
    """Time every candidate (`candidates`) on `scene` with `cams` and the
    device `targets` (float3 per pixel, as Trainer.set_targets takes), and
    return `base` with the fastest one's tile shape and binning path, plus
    every trial.  A candidate the library rejects (a tile shape that does not
    fit its blend kernel, an allocation that fails) is recorded with its
    error and skipped; if none runs, RuntimeError."""
    trials = []
    for cfg in candidates(base, tiles, sort_modes):
        try:
            ms = timer(ctx, scene, cams, targets, cfg, warmup, steps)
            trials.append(Trial(cfg.tile_w, cfg.tile_h, cfg.sort_mode, float(ms), None))
        except SplatCudaError as e:
            trials.append(Trial(cfg.tile_w, cfg.tile_h, cfg.sort_mode, None, str(e)))
    b = trials[pick(trials)]
    return replace(base, tile_w=b.tile_w, tile_h=b.tile_h, sort_mode=b.sort_mode), trials
