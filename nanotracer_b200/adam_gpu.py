"""Optimiser — the mirror of AdamConfig / AdamGpu (crates/nano-optimize/src/adam.rs:22-39,
adam_gpu.rs:31-547) and of the densify / prune steps of train.rs:414-602, run
on the device by stream compaction in the reference's swap_remove order.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import check, lib, sc_adam_config, sc_adam_groups
from .gpu import CudaCtx, DeviceBuffer
from .splat_gpu import AdamMomentBuffers, GpuSplatBuffer, GradSplatBuffers

# train.rs:37-39
LOG_SCALE_MIN = -10.0
LOG_SCALE_MAX = 5.0
OPACITY_LOGIT_MAX = 10.0
# train.rs:103-114
PRUNE_EVERY = 100
PRUNE_WARMUP = 50
PRUNE_OPACITY_LOGIT = -5.3
DENSIFY_EVERY = 200
DENSIFY_WARMUP = 100
DENSIFY_GRAD_THRESHOLD = 2e-4
SPLIT_SCALE_THRESHOLD = -2.3


@dataclass
class AdamConfig:
    lr: float = 1.6e-4
    beta1: float = 0.9
    beta2: float = 0.999
    eps: float = 1e-15

    def struct(self) -> sc_adam_config:
        return sc_adam_config(self.lr, self.beta1, self.beta2, self.eps)


def adam_groups(lrs, beta1=0.9, beta2=0.999, eps=1e-15) -> sc_adam_groups:
    g = sc_adam_groups()
    for i, v in enumerate(lrs):
        g.lr[i] = float(v)
    g.beta1, g.beta2, g.eps = beta1, beta2, eps
    return g


class AdamGpu:
    def __init__(self, ctx: CudaCtx):
        self.ctx = ctx

    def step(self, params: DeviceBuffer, grads: DeviceBuffer, m: DeviceBuffer, v: DeviceBuffer, n_scalars: int,
             lr: float, t: int, cfg: AdamConfig) -> None:
        c = cfg.struct()
        check(lib().sc_adam_step(self.ctx.handle, params.cptr, grads.cptr, m.cptr, v.cptr, int(n_scalars), float(lr),
                                 int(t), C.byref(c)), self.ctx.handle)

    def step_all(self, splats: GpuSplatBuffer, grads: GradSplatBuffers, moments: AdamMomentBuffers, t: int,
                 cfg_pos: AdamConfig, cfg_attr: AdamConfig | None = None, lrs=None) -> None:
        """Reference two-group form (pos vs the rest, adam_gpu.rs:334-427) or six explicit lrs."""
        if lrs is None:
            a = cfg_attr or cfg_pos
            lrs = [cfg_pos.lr, a.lr, a.lr, a.lr, a.lr, a.lr]
        g = adam_groups(lrs, cfg_pos.beta1, cfg_pos.beta2, cfg_pos.eps)
        check(lib().sc_adam_step_all(self.ctx.handle, splats.handle, grads.handle, moments.handle, int(t), C.byref(g)),
              self.ctx.handle)

    def apply_constraints(self, splats: GpuSplatBuffer, log_scale_min: float = LOG_SCALE_MIN,
                          log_scale_max: float = LOG_SCALE_MAX, opacity_logit_max: float = OPACITY_LOGIT_MAX) -> None:
        check(lib().sc_apply_constraints(self.ctx.handle, splats.handle, float(log_scale_min), float(log_scale_max),
                                         float(opacity_logit_max)), self.ctx.handle)

    def accumulate_grad(self, grads: GradSplatBuffers, grad_acc: DeviceBuffer, n: int) -> None:
        check(lib().sc_accumulate_grad(self.ctx.handle, grads.handle, grad_acc.cptr, int(n)), self.ctx.handle)

    def zero_grad_acc(self, grad_acc: DeviceBuffer) -> None:
        grad_acc.zero()


def prune_low_opacity(ctx: CudaCtx, splats: GpuSplatBuffer, moments: AdamMomentBuffers | None,
                      grad_acc: DeviceBuffer | None, threshold: float = PRUNE_OPACITY_LOGIT) -> int:
    removed = C.c_uint32()
    check(lib().sc_prune_low_opacity(ctx.handle, splats.handle, moments.handle if moments else None,
                                     grad_acc.cptr if grad_acc is not None else None, float(threshold),
                                     C.byref(removed)), ctx.handle)
    return removed.value


def densify(ctx: CudaCtx, splats: GpuSplatBuffer, moments: AdamMomentBuffers | None, grad_acc: DeviceBuffer,
            grad_count: int, grad_threshold: float = DENSIFY_GRAD_THRESHOLD,
            split_log_scale_threshold: float = SPLIT_SCALE_THRESHOLD, max_splats: int = 6_000_000,
            it: int = 0) -> tuple[int, int, int]:
    counts = (C.c_uint32 * 3)()
    check(lib().sc_densify(ctx.handle, splats.handle, moments.handle if moments else None, grad_acc.cptr,
                           int(grad_count), float(grad_threshold), float(split_log_scale_threshold), int(max_splats),
                           int(it), counts), ctx.handle)
    return counts[0], counts[1], counts[2]
