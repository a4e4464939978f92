"""Data-parallel views: one training iteration split across ranks by views.

The reference trains on one device: train.rs:155-250 renders an iteration's
views one after another and steps Adam once.  Here each of R ranks (one
process per GPU, torch.distributed over NCCL) takes a block of the views and
the iteration runs ZeRO-1 style, with one exchange in each direction:

  1. every rank renders and back-propagates its views and sums the per-splat
     gradient over them, written shard-major (chunks of `shard` splats, each
     chunk 59 rows x shard) -- sc_trainer_step_grads;
  2. reduce-scatter of that buffer: rank r receives the summed chunk r;
  3. Adam + densify statistic + constraints on splats [r*shard, r*shard+count)
     -- sc_adam_step_shard;
  4. the chunk's updated parameters are packed (sc_splats_pack_range),
     all-gathered, and unpacked on every rank (sc_splats_unpack_shards).

Every rank holds the full parameters (they are what it renders) and full-size
moment and statistic buffers, of which it updates only its own chunk.  Before a
densify or prune (train.rs:259-362) the chunks of the moments and of the
densify statistic are all-gathered, then every rank runs the same device
compaction on identical inputs, so the stores stay identical without a
broadcast.

The loss is the mean over all views of the iteration: each rank scales dL/dC
and its loss by 1/V_total and the losses are summed across ranks.

ViewParallelTrainer holds the sharding arithmetic and the collective sequence;
the per-rank compute is a backend object.  CudaViewBackend is the product
backend (the C ABI on this rank's GPU); tests drive the same trainer with a
CPU backend over gloo.
"""
from __future__ import annotations

import ctypes as C
from typing import Protocol, Sequence

import numpy as np

PARAM_ROWS = 59
SHARD_ALIGN = 64  # splats per chunk rounded up to this (128-byte chunk rows)


# ---------------------------------------------------------------- sharding arithmetic
def shard_size(n: int, world: int, align: int = SHARD_ALIGN) -> int:
    """Splats per chunk: ceil(n / world) rounded up to `align`, at least `align`."""
    per = -(-max(n, 1) // world)
    return max(align, -(-per // align) * align)


def chunk_range(n: int, shard: int, rank: int) -> tuple[int, int]:
    """(lo, count) of the splats rank `rank` updates; count may be 0 for trailing ranks."""
    lo = min(rank * shard, n)
    return lo, max(0, min(shard, n - lo))


def split_views(total: int, world: int, rank: int) -> list[int]:
    """Contiguous block of view indices for `rank`; the first total % world ranks take one more."""
    base, rem = divmod(total, world)
    lo = rank * base + min(rank, rem)
    return list(range(lo, lo + base + (1 if rank < rem else 0)))


class ViewBackend(Protocol):
    """Per-rank compute that ViewParallelTrainer drives (buffers are torch tensors
    on the backend's device)."""

    n: int

    def step_grads(self, views: Sequence[int], loss_weight: float, n_shards: int, shard: int, grads) -> float: ...
    def adam_shard(self, chunk, lo: int, count: int, shard: int, t: int) -> None: ...
    def pack_params(self, lo: int, count: int, shard: int, out) -> None: ...
    def unpack_params(self, gathered, n_shards: int, shard: int) -> None: ...
    def pack_moments(self, lo: int, count: int, shard: int, out) -> None: ...
    def unpack_moments(self, gathered, n_shards: int, shard: int) -> None: ...
    def grad_acc(self): ...
    def densify_prune(self, it: int, grad_count: int, do_prune: bool, do_densify: bool) -> None: ...
    def stream_context(self): ...


class ViewParallelTrainer:
    """The split iteration over a process group (torch.distributed)."""

    def __init__(self, backend: ViewBackend, total_views: int, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.be = backend
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.total_views = total_views
        self.views = split_views(total_views, self.world, self.rank)
        if not self.views:
            raise ValueError(f"rank {self.rank} has no views: {total_views} views over {self.world} ranks")
        self._bufs: dict[str, object] = {}

    # -- buffers (reused while the splat count fits)
    def _buf(self, name: str, numel: int):
        import torch
        b = self._bufs.get(name)
        if b is None or b.numel() < numel:
            with self.be.stream_context():  # filled on the stream that uses it
                b = torch.zeros(numel, dtype=torch.float32, device=self.be.device)
            self._bufs[name] = b
        return b[:numel]

    def plan(self) -> tuple[int, int, int]:
        """(shard, lo, count) for the current splat count."""
        shard = shard_size(self.be.n, self.world)
        lo, count = chunk_range(self.be.n, shard, self.rank)
        return shard, lo, count

    def step(self, t: int) -> float:
        """One iteration (Adam step t, 1-based); returns the loss over all views."""
        import torch
        dist, R = self.dist, self.world
        shard, lo, count = self.plan()
        rows = PARAM_ROWS * shard
        grads = self._buf("grads", R * rows)
        chunk = self._buf("chunk", rows)
        send = self._buf("send", rows)
        gathered = self._buf("gathered", R * rows)
        loss_local = self.be.step_grads(self.views, 1.0 / self.total_views, R, shard, grads)
        with self.be.stream_context():
            dist.reduce_scatter_tensor(chunk, grads, op=dist.ReduceOp.SUM, group=self.group)
            self.be.adam_shard(chunk, lo, count, shard, t)
            self.be.pack_params(lo, count, shard, send)
            dist.all_gather_into_tensor(gathered, send, group=self.group)
            self.be.unpack_params(gathered, R, shard)
            loss = torch.tensor([loss_local], dtype=torch.float64, device=self.be.device)
            dist.all_reduce(loss, op=dist.ReduceOp.SUM, group=self.group)
        return float(loss.item())

    def gather_state(self) -> None:
        """Give every rank the full moments and densify statistic (before a densify/prune)."""
        dist, R = self.dist, self.world
        shard, lo, count = self.plan()
        send = self._buf("msend", 2 * PARAM_ROWS * shard)
        gathered = self._buf("mgathered", R * 2 * PARAM_ROWS * shard)
        acc = self.be.grad_acc()
        acc_send = self._buf("asend", shard)
        acc_all = self._buf("aall", R * shard)
        with self.be.stream_context():
            self.be.pack_moments(lo, count, shard, send)
            dist.all_gather_into_tensor(gathered, send, group=self.group)
            self.be.unpack_moments(gathered, R, shard)
            acc_send.zero_()
            acc_send[:count].copy_(acc[lo:lo + count])
            dist.all_gather_into_tensor(acc_all, acc_send, group=self.group)
            acc[: self.be.n].copy_(acc_all[: self.be.n])

    def maybe_densify(self, it: int, grad_count: int, prune_warmup: int, prune_every: int, densify_warmup: int,
                      densify_every: int) -> bool:
        """train.rs:259-362 schedule; returns True when the densify statistic was reset."""
        do_prune = it >= prune_warmup and it % prune_every == 0
        do_densify = it >= densify_warmup and it % densify_every == 0 and grad_count > 0
        if not (do_prune or do_densify):
            return False
        self.gather_state()
        self.be.densify_prune(it, grad_count, do_prune, do_densify)
        return do_densify

    def close(self) -> None:
        self._bufs.clear()


# ---------------------------------------------------------------- CUDA backend
class CudaViewBackend:
    """This rank's GPU through the C ABI: a batched sc_trainer for its views, the
    splat store, moments and densify statistic.  Buffers exchanged with NCCL are
    torch tensors whose device pointers go to the library; the collectives run
    on the library context's stream (wrapped as a torch ExternalStream), so they
    are ordered with the kernels without extra synchronisation."""

    def __init__(self, ctx, splats, cfg, targets_all: np.ndarray, views: Sequence[int], max_splats: int | None = None):
        import torch
        from .splat_gpu import AdamMomentBuffers, GpuSplatBuffer
        from .train import Trainer, TrainConfig
        self.torch = torch
        self.ctx = ctx
        self.device = torch.device("cuda", ctx.device)
        torch.cuda.set_device(self.device)
        self.ext_stream = torch.cuda.ExternalStream(ctx.stream, device=self.device)
        self.cfg = cfg
        cap = max(max_splats or len(splats), len(splats))
        self.g = GpuSplatBuffer.upload(ctx, splats, capacity=cap, bf16_rest=cfg.bf16)
        self.mo = AdamMomentBuffers(ctx, self.g.capacity, bf16=cfg.bf16)
        self.acc = torch.zeros(self.g.capacity, dtype=torch.float32, device=self.device)
        local = TrainConfig(**{**cfg.__dict__, "n_views": len(views)})
        self.trainer = Trainer(ctx, local)
        tg = np.ascontiguousarray(np.asarray(targets_all, np.float32)[list(views)])
        self.targets = ctx.storage_buffer("targets", tg)
        self.trainer.set_targets(self.targets)
        self._cams = None

    @property
    def n(self) -> int:
        return self.g.n

    def set_cameras(self, cams) -> None:
        """This rank's cameras for the next step (its views only)."""
        self._cams = cams

    def stream_context(self):
        return self.torch.cuda.stream(self.ext_stream)

    def _lib(self):
        from ._lib import lib
        return lib()

    def _check(self, st):
        from ._lib import check
        check(st, self.ctx.handle)

    @staticmethod
    def _ptr(t) -> C.c_void_p:
        return C.c_void_p(t.data_ptr())

    def step_grads(self, views, loss_weight, n_shards, shard, grads) -> float:
        from .raster import cameras_array
        if self._cams is None or len(self._cams) != len(views):
            raise ValueError("set_cameras() with one camera per local view before step()")
        loss = C.c_double()
        # the library stream must not run ahead of torch work that produced `grads`' storage
        self.ext_stream.wait_stream(self.torch.cuda.current_stream(self.device))
        self._check(self._lib().sc_trainer_step_grads(self.trainer.handle, self.g.handle, cameras_array(self._cams),
                                                      C.c_float(loss_weight), n_shards, shard, self._ptr(grads),
                                                      C.byref(loss)))
        return loss.value

    def adam_shard(self, chunk, lo, count, shard, t) -> None:
        from .adam_gpu import LOG_SCALE_MAX, LOG_SCALE_MIN, OPACITY_LOGIT_MAX, adam_groups
        c = self.cfg
        gr = adam_groups(c.lrs, c.beta1, c.beta2, c.eps)
        self._check(self._lib().sc_adam_step_shard(self.ctx.handle, self.g.handle, self.mo.handle,
                                                   self._ptr(self.acc), self._ptr(chunk), lo, count, shard, int(t),
                                                   C.byref(gr), LOG_SCALE_MIN, LOG_SCALE_MAX, OPACITY_LOGIT_MAX))

    def pack_params(self, lo, count, shard, out) -> None:
        self._check(self._lib().sc_splats_pack_range(self.ctx.handle, self.g.handle, lo, count, shard, self._ptr(out)))

    def unpack_params(self, gathered, n_shards, shard) -> None:
        self._check(self._lib().sc_splats_unpack_shards(self.ctx.handle, self.g.handle, self._ptr(gathered),
                                                        n_shards, shard))

    def pack_moments(self, lo, count, shard, out) -> None:
        self._check(self._lib().sc_moments_pack_range(self.ctx.handle, self.mo.handle, lo, count, shard,
                                                      self._ptr(out)))

    def unpack_moments(self, gathered, n_shards, shard) -> None:
        self._check(self._lib().sc_moments_unpack_shards(self.ctx.handle, self.mo.handle, self.g.n,
                                                         self._ptr(gathered), n_shards, shard))

    def grad_acc(self):
        return self.acc

    def densify_prune(self, it, grad_count, do_prune, do_densify) -> None:
        from .adam_gpu import (DENSIFY_GRAD_THRESHOLD, PRUNE_OPACITY_LOGIT, SPLIT_SCALE_THRESHOLD, densify,
                               prune_low_opacity)
        acc = _TensorBuffer(self.acc)
        if do_prune:
            prune_low_opacity(self.ctx, self.g, self.mo, acc, PRUNE_OPACITY_LOGIT)
        if do_densify:
            densify(self.ctx, self.g, self.mo, acc, grad_count, DENSIFY_GRAD_THRESHOLD, SPLIT_SCALE_THRESHOLD,
                    min(self.cfg.max_splats, self.g.capacity), it)
            with self.stream_context():
                self.acc.zero_()

    def images(self) -> np.ndarray:
        return self.trainer.images()


class _TensorBuffer:
    """A torch CUDA tensor seen as a library buffer (the .cptr the wrappers pass)."""

    def __init__(self, t):
        self.t = t

    @property
    def cptr(self) -> C.c_void_p:
        return C.c_void_p(self.t.data_ptr())

    @property
    def nbytes(self) -> int:
        return self.t.numel() * self.t.element_size()

    def zero(self) -> None:
        self.t.zero_()


def expected_shards(n: int, world: int) -> list[tuple[int, int]]:
    """(lo, count) of every rank; the chunks tile [0, n) exactly."""
    shard = shard_size(n, world)
    return [chunk_range(n, shard, r) for r in range(world)]
