"""Many scenes in one launch per stage — no counterpart in the reference,
whose train() (crates/nano-optimize/src/train.rs:65-401) trains one scene per
call.

ScenesTrainer wraps sc_scenes_trainer: n scenes, each with its own splat
store, Adam moments, densify statistic, camera, image size and target, are
stepped together, every stage one launch over all scenes and the whole step
one CUDA graph.  Images of different sizes share a tile grid of the largest
size.  Densify and prune stay per scene (the reference's schedule and rules,
train.rs:103-114, 259-362) on each scene's own store, through
adam_gpu.densify / prune_low_opacity; train_scenes() runs that schedule with
a cap on the total splat count.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import check, lib, sc_scenes_config
from .adam_gpu import (DENSIFY_GRAD_THRESHOLD, LOG_SCALE_MAX, LOG_SCALE_MIN, OPACITY_LOGIT_MAX, PRUNE_OPACITY_LOGIT,
                       SPLIT_SCALE_THRESHOLD, adam_groups, densify, prune_low_opacity)
from .gpu import CudaCtx, DeviceBuffer
from .raster import CameraUniform, cameras_array
from .splat_gpu import AdamMomentBuffers, GpuSplatBuffer
from .splat_store import SplatBuffer
from .train import BENCH_LRS


@dataclass
class Scene:
    """One scene's device state and image."""
    splats: GpuSplatBuffer
    moments: AdamMomentBuffers
    grad_acc: DeviceBuffer
    width: int
    height: int
    target: DeviceBuffer  # width * height float3

    @classmethod
    def upload(cls, ctx: CudaCtx, splats: SplatBuffer, target: np.ndarray, capacity: int = 0) -> "Scene":
        g = GpuSplatBuffer.upload(ctx, splats, capacity=capacity)
        mo = AdamMomentBuffers(ctx, g.capacity)
        acc = ctx.storage_buffer_zeroed("grad_acc", 4 * g.capacity)
        h, w = target.shape[:2]
        return cls(g, mo, acc, w, h, ctx.storage_buffer("target", np.ascontiguousarray(target, np.float32)))


class ScenesTrainer:
    def __init__(self, ctx: CudaCtx, n_scenes: int, max_width: int, max_height: int, tile: int = 16,
                 lrs=BENCH_LRS, use_graph: bool = True, tile_cull: bool = True, depth_max: float = 8.0):
        self.ctx = ctx
        self.n, self.max_width, self.max_height = n_scenes, max_width, max_height
        c = sc_scenes_config()
        c.n_scenes = n_scenes
        c.tiling.width, c.tiling.height = max_width, max_height
        c.tiling.tile_w = c.tiling.tile_h = tile
        c.tiling.depth_max = depth_max
        c.adam = adam_groups(lrs, 0.9, 0.999, 1e-15)
        c.use_graph = 1 if use_graph else 0
        c.tile_cull = 1 if tile_cull else 0
        c.log_scale_min, c.log_scale_max, c.opacity_logit_max = LOG_SCALE_MIN, LOG_SCALE_MAX, OPACITY_LOGIT_MAX
        h = C.c_void_p()
        check(lib().sc_scenes_trainer_create(ctx.handle, C.byref(c), C.byref(h)), ctx.handle)
        self.handle = h
        self.scenes: list[Scene | None] = [None] * n_scenes

    def set_scene(self, i: int, scene: Scene) -> None:
        self.scenes[i] = scene
        check(lib().sc_scenes_trainer_set_scene(self.handle, i, scene.splats.handle, scene.moments.handle,
                                                scene.grad_acc.cptr, scene.width, scene.height, scene.target.cptr),
              self.ctx.handle)

    def step(self, cams: list[CameraUniform], t: int) -> np.ndarray:
        losses = (C.c_double * self.n)()
        check(lib().sc_scenes_trainer_step(self.handle, cameras_array(cams), int(t), losses), self.ctx.handle)
        return np.array(losses[:], np.float64)

    def images(self) -> list[np.ndarray]:
        """Each scene's image of the last step (height, width, 4)."""
        p = C.c_void_p()
        check(lib().sc_scenes_trainer_images(self.handle, C.byref(p)), self.ctx.handle)
        full = np.empty(self.n * self.max_height * self.max_width * 4, np.float32)
        check(lib().sc_buffer_readback(self.ctx.handle, C.c_void_p(full.ctypes.data), p, full.nbytes),
              self.ctx.handle)
        full = full.reshape(self.n, self.max_height, self.max_width, 4)
        return [full[i, :s.height, :s.width] for i, s in enumerate(self.scenes)]

    def stats(self) -> dict:
        pairs, nk, items = C.c_uint64(), C.c_uint32(), C.c_uint64()
        check(lib().sc_scenes_trainer_stats(self.handle, C.byref(pairs), C.byref(nk), C.byref(items)),
              self.ctx.handle)
        return {"pairs": pairs.value, "items": items.value, "kernels_per_step": nk.value}

    def close(self) -> None:
        if self.handle and self.ctx.handle:
            lib().sc_scenes_trainer_free(self.ctx.handle, self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def densify_prune_scenes(trainer: ScenesTrainer, it: int, grad_count: int, max_total: int,
                         prune_every: int = 100, prune_warmup: int = 50, densify_every: int = 200,
                         densify_warmup: int = 100) -> dict:
    """The reference's prune / densify schedule (train.rs:259-362) per scene
    after step `it`, with the densify budget max_total shared by the scenes:
    a scene may grow by at most its share of the room left (the total splat
    count never exceeds max_total, nor a scene its store's capacity).
    Returns per-event counts."""
    out = {"pruned": 0, "cloned": 0, "split": 0}
    if it >= prune_warmup and it % prune_every == 0:
        for s in trainer.scenes:
            out["pruned"] += prune_low_opacity(trainer.ctx, s.splats, s.moments, s.grad_acc, PRUNE_OPACITY_LOGIT)
    if it >= densify_warmup and it % densify_every == 0:
        total = sum(s.splats.n for s in trainer.scenes)
        room = max(0, max_total - total)
        for s in trainer.scenes:
            share = room // len(trainer.scenes)
            cap = min(s.splats.capacity, s.splats.n + share)
            c = densify(trainer.ctx, s.splats, s.moments, s.grad_acc, grad_count, DENSIFY_GRAD_THRESHOLD,
                        SPLIT_SCALE_THRESHOLD, cap, it)
            out["cloned"] += c[0]
            out["split"] += c[1]
            s.grad_acc.zero()
    return out
