"""Checkpoint and resume of a training run.

The splats go to the reference's Inria PLY (crates/nano-splat/src/ply.rs:17-256,
through the library's writer); next to it, `<path>.adam.npz` holds what the
PLY cannot: the Adam moments m and v in the same splat order and the shared
step count t (adam.rs:48-56, train.rs:229), and the densify statistic with its
sample count (train.rs:322-326).  The reference keeps none of this across runs
(its roadmap lists it next to the PLY writer); a run resumed from a checkpoint
continues with the same parameters, moments and bias corrections.

All parameter and moment values round-trip bit for bit (f32 on disk; bf16
device forms widen exactly and round back to the same value).
"""
from __future__ import annotations

from dataclasses import dataclass
from pathlib import Path

import numpy as np

from .ply import read_ply, write_ply
from .splat_store import SplatBuffer

MAGIC = "nanotracer-adam-v1"


def sidecar(path: str | Path) -> Path:
    return Path(str(path) + ".adam.npz")


@dataclass
class Checkpoint:
    splats: SplatBuffer
    m: SplatBuffer
    v: SplatBuffer
    t: int
    grad_acc: np.ndarray
    grad_count: int


def save_checkpoint(path: str | Path, splats: SplatBuffer, m: SplatBuffer, v: SplatBuffer, t: int,
                    grad_acc: np.ndarray | None = None, grad_count: int = 0) -> None:
    n = len(splats)
    if len(m) != n or len(v) != n:
        raise ValueError(f"moments hold {len(m)}/{len(v)} splats, the store {n}")
    acc = np.zeros(n, np.float32) if grad_acc is None else np.ascontiguousarray(grad_acc[:n], np.float32)
    if acc.shape != (n,):
        raise ValueError("grad_acc must hold one value per splat")
    write_ply(path, splats)
    np.savez(sidecar(path), magic=np.array(MAGIC), n=np.int64(n), t=np.int64(t), m=m.flat(), v=v.flat(),
             grad_acc=acc, grad_count=np.int64(grad_count))


def load_checkpoint(path: str | Path) -> Checkpoint:
    splats = read_ply(path)
    with np.load(sidecar(path)) as z:
        if str(z["magic"]) != MAGIC:
            raise ValueError(f"{sidecar(path)}: not a {MAGIC} sidecar")
        n = int(z["n"])
        if n != len(splats):
            raise ValueError(f"{sidecar(path)} holds {n} splats, the PLY {len(splats)}")
        return Checkpoint(splats, SplatBuffer.from_flat(z["m"]), SplatBuffer.from_flat(z["v"]), int(z["t"]),
                          np.array(z["grad_acc"], np.float32), int(z["grad_count"]))


def save_device_checkpoint(path: str | Path, ctx, splats, moments, grad_acc, t: int, grad_count: int = 0) -> None:
    """Read back a device store (GpuSplatBuffer), its AdamMomentBuffers and the
    densify-statistic buffer, and write the checkpoint."""
    n = splats.n
    m, v = moments.download(n)
    acc = grad_acc.readback(np.float32, n) if grad_acc is not None else None
    save_checkpoint(path, splats.readback(), m, v, t, acc, grad_count)


def load_device_checkpoint(path: str | Path, ctx, capacity: int = 0, bf16: bool = False):
    """Upload a checkpoint: returns (GpuSplatBuffer, AdamMomentBuffers, grad_acc DeviceBuffer, t, grad_count)."""
    from .splat_gpu import AdamMomentBuffers, GpuSplatBuffer
    ck = load_checkpoint(path)
    g = GpuSplatBuffer.upload(ctx, ck.splats, capacity=capacity, bf16_rest=bf16)
    mo = AdamMomentBuffers.upload_from_cpu(ctx, ck.m, ck.v, g.capacity, bf16)
    acc = ctx.storage_buffer_zeroed("grad_acc", 4 * g.capacity)
    if len(ck.grad_acc):
        acc.upload(ck.grad_acc)
    return g, mo, acc, ck.t, ck.grad_count
