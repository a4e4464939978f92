"""Training driver — the mirror of nano-optimize's train()
(crates/nano-optimize/src/train.rs:37-401) on the batched device trainer.

Trainer wraps sc_trainer: one step = n_views views (project -> bin -> blend
-> MSE dL/dC -> backward -> project backward summed over views -> grad
accumulation -> Adam -> constraints) replayed as one CUDA graph.  train()
adds the reference's schedule around it: prune every 100 iterations after 50,
densify every 200 after 100 (train.rs:103-114, 259-362), both on the device.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from ._lib import SC_BWD_EXACT, SC_BWD_REF, check, lib, sc_camera, sc_train_config
from .adam_gpu import (DENSIFY_EVERY, DENSIFY_GRAD_THRESHOLD, DENSIFY_WARMUP, LOG_SCALE_MAX, LOG_SCALE_MIN,
                       OPACITY_LOGIT_MAX, PRUNE_EVERY, PRUNE_OPACITY_LOGIT, PRUNE_WARMUP, SPLIT_SCALE_THRESHOLD,
                       AdamConfig, adam_groups, densify, prune_low_opacity)
from .gpu import CudaCtx, DeviceBuffer
from .raster import CameraUniform, cameras_array
from .splat_gpu import AdamMomentBuffers, GpuSplatBuffer
from .splat_store import SplatBuffer
from .tile_binner import TilingParams

# per-group learning rates used for the synthetic benchmark scenes:
# means, rotation, scale, opacity, SH DC, SH rest
BENCH_LRS = (1.6e-4, 1e-3, 5e-3, 0.05, 2.5e-3, 1.25e-4)


@dataclass
class TrainConfig:
    iterations: int = 100
    max_splats: int = 6_000_000
    n_views: int = 1
    width: int = 256
    height: int = 256
    tile_w: int = 16
    tile_h: int = 16
    depth_max: float = 8.0
    lrs: tuple = BENCH_LRS
    beta1: float = 0.9
    beta2: float = 0.999
    eps: float = 1e-15
    exact_backward: bool = True
    use_graph: bool = True
    densify: bool = True
    bf16: bool = False
    tile_cull: bool = True
    ssim_lambda: float = 0.0
    sort_mode: int = 0  # 0 auto (two-level binning), 1 sort of the (tile, splat) pairs, 2 two-level
    fp64_det: bool = False  # FP64 determinant / inverse of near-degenerate splats (projection and adjoint)
    compensated_sums: bool = False  # TwoSum-compensated per-(view, splat) gradient totals across tiles
    blend_batch: int = 0  # list positions staged per blend batch (multiple of 32); 0 = one per thread
    sort_digit_bits: int = 0  # radix digit width of the binning sort: 8, 9, or 0 = fewer passes wins

    def struct(self) -> sc_train_config:
        c = sc_train_config()
        c.n_views = self.n_views
        c.tiling.width, c.tiling.height = self.width, self.height
        c.tiling.tile_w, c.tiling.tile_h = self.tile_w, self.tile_h
        c.tiling.depth_max = self.depth_max
        c.adam = adam_groups(self.lrs, self.beta1, self.beta2, self.eps)
        c.bwd_mode = SC_BWD_EXACT if self.exact_backward else SC_BWD_REF
        c.use_graph = 1 if self.use_graph else 0
        c.tile_cull = 1 if self.tile_cull else 0
        c.log_scale_min, c.log_scale_max, c.opacity_logit_max = LOG_SCALE_MIN, LOG_SCALE_MAX, OPACITY_LOGIT_MAX
        c.ssim_lambda = self.ssim_lambda
        c.sort_mode = self.sort_mode
        c.fp64_det = 1 if self.fp64_det else 0
        c.compensated_sums = 1 if self.compensated_sums else 0
        c.blend_batch = self.blend_batch
        c.sort_digit_bits = self.sort_digit_bits
        return c


class Trainer:
    def __init__(self, ctx: CudaCtx, cfg: TrainConfig):
        self.ctx = ctx
        self.cfg = cfg
        c = cfg.struct()
        h = C.c_void_p()
        check(lib().sc_trainer_create(ctx.handle, C.byref(c), C.byref(h)), ctx.handle)
        self.handle = h
        self._targets = None

    def set_targets(self, targets: DeviceBuffer) -> None:
        self._targets = targets
        check(lib().sc_trainer_set_targets(self.handle, targets.cptr), self.ctx.handle)

    def set_host_targets(self, pinned_ptr: int, keepalive=None) -> None:
        """Targets in page-locked host memory at `pinned_ptr`; copied on a side
        stream every step, overlapped with the stages before the blend."""
        self._targets = keepalive
        check(lib().sc_trainer_set_host_targets(self.handle, C.c_void_p(pinned_ptr)), self.ctx.handle)

    def set_profiling(self, on: bool | int) -> None:
        """False/0 off; True/1 stage times and blend work; 2 also the blends'
        (pixel, entry) pair counts.  Each call resets the accumulators."""
        level = int(on) if not isinstance(on, bool) else (1 if on else 0)
        check(lib().sc_trainer_set_profiling(self.handle, level), self.ctx.handle)

    def step(self, splats: GpuSplatBuffer, moments: AdamMomentBuffers, grad_acc: DeviceBuffer,
             cams: list[CameraUniform], t: int) -> float:
        arr = cameras_array(cams)
        loss = C.c_double()
        check(lib().sc_trainer_step(self.handle, splats.handle, moments.handle, grad_acc.cptr, arr, int(t),
                                    C.byref(loss)), self.ctx.handle)
        return loss.value

    def images_ptr(self) -> int:
        p = C.c_void_p()
        check(lib().sc_trainer_images(self.handle, C.byref(p)), self.ctx.handle)
        return p.value

    def images(self) -> np.ndarray:
        n = self.cfg.n_views * self.cfg.width * self.cfg.height * 4
        out = np.empty(n, np.float32)
        check(lib().sc_buffer_readback(self.ctx.handle, C.c_void_p(out.ctypes.data), C.c_void_p(self.images_ptr()),
                                       out.nbytes), self.ctx.handle)
        return out.reshape(self.cfg.n_views, self.cfg.height, self.cfg.width, 4)

    def stats(self) -> dict:
        pairs, nk, items = C.c_uint64(), C.c_uint32(), C.c_uint64()
        names = (C.c_char_p * 9)()
        ms = (C.c_float * 9)()
        check(lib().sc_trainer_stats(self.handle, C.byref(pairs), C.byref(nk), names, ms, C.byref(items)),
              self.ctx.handle)
        work = (C.c_uint64 * 4)()
        check(lib().sc_trainer_blend_work(self.handle, work), self.ctx.handle)
        px = (C.c_uint64 * 2)()
        check(lib().sc_trainer_blend_pairs(self.handle, px), self.ctx.handle)
        return {"pairs": pairs.value, "items": items.value, "kernels_per_step": nk.value,
                "stage_ms": {names[i].decode(): float(ms[i]) for i in range(9)},
                "blend_work": {"fwd_scanned": work[0], "fwd_blended": work[1], "bwd_scanned": work[2],
                               "bwd_blended": work[3], "fwd_pixel_pairs": px[0], "bwd_pixel_pairs": px[1]}}

    def __del__(self):
        try:
            if self.handle and self.ctx.handle:
                lib().sc_trainer_free(self.ctx.handle, self.handle)
                self.handle = None
        except Exception:
            pass


def render_targets(ctx: CudaCtx, scene: SplatBuffer, cams: list[CameraUniform], tiling: TilingParams) -> np.ndarray:
    """Render float3 target images of `scene` from `cams` with the device path (synthetic ground truth)."""
    from .raster import Rasterizer
    from .tile_binner import TileBinner
    from ._lib import SC_KEYS_NATIVE64
    g = GpuSplatBuffer.upload(ctx, scene)
    r, b = Rasterizer(ctx), TileBinner(ctx)
    V = len(cams)
    proj = r.alloc_projected(g, V)
    r.project(g, cams, proj)
    bins = b.bin(proj, len(scene), tiling, stride=g.capacity, n_views=V, key_mode=SC_KEYS_NATIVE64)
    img = r.alloc_image(tiling.width, tiling.height, V)
    r.composite(proj, bins, img, tiling, stride=g.capacity, n_views=V)
    out = img.readback(np.float32).reshape(V, tiling.height, tiling.width, 4)
    return np.ascontiguousarray(out[..., :3])


def train(ctx: CudaCtx, splats: SplatBuffer, targets: np.ndarray, poses_fn, cfg: TrainConfig, on_iter=None):
    """train.rs:65-401 with a host-supplied view schedule: poses_fn(iter) -> list of
    CameraUniform for that step; targets (n_views, H, W, 3) or a callable iter -> targets.
    Returns the final SplatBuffer."""
    cap = max(cfg.max_splats, len(splats)) if cfg.densify else len(splats)
    g = GpuSplatBuffer.upload(ctx, splats, capacity=cap, bf16_rest=cfg.bf16)
    mo = AdamMomentBuffers(ctx, g.capacity, bf16=cfg.bf16)
    acc = ctx.storage_buffer_zeroed("grad_acc", g.capacity * 4)
    tr = Trainer(ctx, cfg)
    tbuf = None
    grad_count = 0
    for it in range(cfg.iterations):
        tg = targets(it) if callable(targets) else targets
        if tbuf is None or tbuf.nbytes != tg.nbytes:
            tbuf = ctx.storage_buffer("targets", np.ascontiguousarray(tg, np.float32))
            tr.set_targets(tbuf)
        elif callable(targets):
            tbuf.upload(np.ascontiguousarray(tg, np.float32))
        loss = tr.step(g, mo, acc, poses_fn(it), it + 1)
        grad_count += 1
        if cfg.densify:
            do_prune = it >= PRUNE_WARMUP and it % PRUNE_EVERY == 0
            do_densify = it >= DENSIFY_WARMUP and it % DENSIFY_EVERY == 0
            if do_prune:
                prune_low_opacity(ctx, g, mo, acc, PRUNE_OPACITY_LOGIT)
            if do_densify and grad_count > 0:
                densify(ctx, g, mo, acc, grad_count, DENSIFY_GRAD_THRESHOLD, SPLIT_SCALE_THRESHOLD, cfg.max_splats, it)
                acc.zero()
                grad_count = 0
        if on_iter is not None:
            on_iter(it, loss, g.n)
    return g.readback()
