"""Data-parallel views: one training iteration split across ranks by views.

The reference trains on one device: train.rs:155-250 renders an iteration's
views one after another and steps Adam once.  Here each of R ranks (one
process per GPU) takes a block of the views and the iteration runs ZeRO-1
style, with one exchange in each direction:

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
the per-rank compute is a backend object and the exchange a collectives
object over the backend's buffers.  The product pair is CudaViewBackend with
CudaCollectives: library device buffers, NCCL through its C API (nccl.py) on
the library context's stream, no other runtime.  Tests drive the same trainer
with an oracle backend and CPU collectives over gloo.
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
    """Per-rank compute that ViewParallelTrainer drives; its buffers are the
    collectives object's."""

    n: int

    def step_grads(self, views: Sequence[int], loss_weight: float, n_shards: int, shard: int, grads) -> float: ...
    def adam_shard(self, chunk, lo: int, count: int, shard: int, t: int) -> None: ...
    def pack_params(self, lo: int, count: int, shard: int, out) -> None: ...
    def unpack_params(self, gathered, n_shards: int, shard: int) -> None: ...
    def pack_moments(self, lo: int, count: int, shard: int, out) -> None: ...
    def unpack_moments(self, gathered, n_shards: int, shard: int) -> None: ...
    def grad_acc(self): ...
    def densify_prune(self, it: int, grad_count: int, do_prune: bool, do_densify: bool) -> None: ...


class Collectives(Protocol):
    """The exchange of one split iteration over float32 buffers of the
    backend's kind (all sums); world and rank of this process."""

    world: int
    rank: int

    def alloc(self, numel: int): ...                      # zero-filled
    def view(self, buf, offset: int, numel: int): ...     # a window into buf
    def zero(self, buf) -> None: ...
    def copy(self, dst, src) -> None: ...                  # same numel
    def reduce_scatter(self, out, inp) -> None: ...        # inp = world chunks of out.numel
    def all_gather(self, out, inp) -> None: ...            # out = world chunks of inp.numel
    def all_reduce_scalar(self, x: float) -> float: ...


class ViewParallelTrainer:
    """The split iteration over a collectives object."""

    def __init__(self, backend: ViewBackend, total_views: int, coll: Collectives):
        self.be = backend
        self.coll = coll
        self.world = coll.world
        self.rank = coll.rank
        self.total_views = total_views
        self.views = split_views(total_views, self.world, self.rank)
        if not self.views:
            raise ValueError(f"rank {self.rank} has no views: {total_views} views over {self.world} ranks")
        self._bufs: dict[str, tuple[object, int]] = {}

    # -- buffers (reused while the splat count fits)
    def _buf(self, name: str, numel: int):
        b = self._bufs.get(name)
        if b is None or b[1] < numel:
            b = (self.coll.alloc(numel), numel)
            self._bufs[name] = b
        return self.coll.view(b[0], 0, numel)

    def plan(self) -> tuple[int, int, int]:
        """(shard, lo, count) for the current splat count."""
        shard = shard_size(self.be.n, self.world)
        lo, count = chunk_range(self.be.n, shard, self.rank)
        return shard, lo, count

    def step(self, t: int) -> float:
        """One iteration (Adam step t, 1-based); returns the loss over all views."""
        R, coll = self.world, self.coll
        shard, lo, count = self.plan()
        rows = PARAM_ROWS * shard
        grads = self._buf("grads", R * rows)
        chunk = self._buf("chunk", rows)
        send = self._buf("send", rows)
        gathered = self._buf("gathered", R * rows)
        loss_local = self.be.step_grads(self.views, 1.0 / self.total_views, R, shard, grads)
        coll.reduce_scatter(chunk, grads)
        self.be.adam_shard(chunk, lo, count, shard, t)
        self.be.pack_params(lo, count, shard, send)
        coll.all_gather(gathered, send)
        self.be.unpack_params(gathered, R, shard)
        return coll.all_reduce_scalar(loss_local)

    def gather_state(self) -> None:
        """Give every rank the full moments and densify statistic (before a densify/prune)."""
        R, coll = self.world, self.coll
        shard, lo, count = self.plan()
        send = self._buf("msend", 2 * PARAM_ROWS * shard)
        gathered = self._buf("mgathered", R * 2 * PARAM_ROWS * shard)
        acc = self.be.grad_acc()
        acc_send = self._buf("asend", shard)
        acc_all = self._buf("aall", R * shard)
        self.be.pack_moments(lo, count, shard, send)
        coll.all_gather(gathered, send)
        self.be.unpack_moments(gathered, R, shard)
        coll.zero(acc_send)
        if count:
            coll.copy(coll.view(acc_send, 0, count), coll.view(acc, lo, count))
        coll.all_gather(acc_all, acc_send)
        if self.be.n:
            coll.copy(coll.view(acc, 0, self.be.n), coll.view(acc_all, 0, self.be.n))

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
class DevBuf:
    """A float32 window of library device memory (an owner buffer keeps it alive)."""

    def __init__(self, ptr: int, numel: int, owner=None):
        self.ptr, self.numel, self.owner = int(ptr), int(numel), owner

    @property
    def cptr(self) -> C.c_void_p:
        return C.c_void_p(self.ptr)

    @property
    def nbytes(self) -> int:
        return 4 * self.numel


class CudaCollectives:
    """Collectives over library device buffers: NCCL (nccl.NcclComm) on the
    library context's stream, device copies and fills through the C ABI on the
    same stream, so the exchange is ordered with the kernels."""

    def __init__(self, ctx, comm):
        self.ctx, self.comm = ctx, comm
        self.world, self.rank = comm.world, comm.rank
        self._scalar = self.alloc(2)

    def alloc(self, numel: int) -> DevBuf:
        from .gpu import DeviceBuffer
        b = DeviceBuffer(self.ctx, 4 * max(int(numel), 1), "collective")
        return DevBuf(b.ptr, numel, b)

    def view(self, buf: DevBuf, offset: int, numel: int) -> DevBuf:
        assert offset + numel <= buf.numel
        return DevBuf(buf.ptr + 4 * offset, numel, buf)

    def zero(self, buf: DevBuf) -> None:
        from ._lib import check, lib
        check(lib().sc_buffer_zero(self.ctx.handle, buf.cptr, buf.nbytes), self.ctx.handle)

    def copy(self, dst: DevBuf, src: DevBuf) -> None:
        from ._lib import check, lib
        assert dst.numel == src.numel
        check(lib().sc_buffer_copy(self.ctx.handle, dst.cptr, src.cptr, dst.nbytes), self.ctx.handle)

    def reduce_scatter(self, out: DevBuf, inp: DevBuf) -> None:
        assert inp.numel == self.world * out.numel
        self.comm.reduce_scatter_f32(out.ptr, inp.ptr, out.numel)

    def all_gather(self, out: DevBuf, inp: DevBuf) -> None:
        assert out.numel == self.world * inp.numel
        self.comm.all_gather_f32(out.ptr, inp.ptr, inp.numel)

    def all_reduce_scalar(self, x: float) -> float:
        from ._lib import check, lib
        v = np.array([x], np.float64)
        check(lib().sc_buffer_upload(self.ctx.handle, self._scalar.cptr, v.ctypes.data_as(C.c_void_p), 8),
              self.ctx.handle)
        self.comm.all_reduce_sum_f64(self._scalar.ptr, 1)
        check(lib().sc_buffer_readback(self.ctx.handle, v.ctypes.data_as(C.c_void_p), self._scalar.cptr, 8),
              self.ctx.handle)
        return float(v[0])


class CudaViewBackend:
    """This rank's GPU through the C ABI: a batched sc_trainer for its views, the
    splat store, moments and densify statistic, all in library memory."""

    def __init__(self, ctx, splats, cfg, targets_all: np.ndarray, views: Sequence[int], max_splats: int | None = None):
        from .splat_gpu import AdamMomentBuffers, GpuSplatBuffer
        from .train import Trainer, TrainConfig
        self.ctx = ctx
        self.cfg = cfg
        cap = max(max_splats or len(splats), len(splats))
        self.g = GpuSplatBuffer.upload(ctx, splats, capacity=cap, bf16_rest=cfg.bf16)
        self.mo = AdamMomentBuffers(ctx, self.g.capacity, bf16=cfg.bf16)
        self._acc = ctx.storage_buffer_zeroed("grad_acc", 4 * self.g.capacity)
        self.acc = DevBuf(self._acc.ptr, self.g.capacity, self._acc)
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

    def _lib(self):
        from ._lib import lib
        return lib()

    def _check(self, st):
        from ._lib import check
        check(st, self.ctx.handle)

    def step_grads(self, views, loss_weight, n_shards, shard, grads: DevBuf) -> float:
        from .raster import cameras_array
        if self._cams is None or len(self._cams) != len(views):
            raise ValueError("set_cameras() with one camera per local view before step()")
        loss = C.c_double()
        self._check(self._lib().sc_trainer_step_grads(self.trainer.handle, self.g.handle, cameras_array(self._cams),
                                                      C.c_float(loss_weight), n_shards, shard, grads.cptr,
                                                      C.byref(loss)))
        return loss.value

    def adam_shard(self, chunk: DevBuf, lo, count, shard, t) -> None:
        from .adam_gpu import LOG_SCALE_MAX, LOG_SCALE_MIN, OPACITY_LOGIT_MAX, adam_groups
        c = self.cfg
        gr = adam_groups(c.lrs, c.beta1, c.beta2, c.eps)
        self._check(self._lib().sc_adam_step_shard(self.ctx.handle, self.g.handle, self.mo.handle, self.acc.cptr,
                                                   chunk.cptr, lo, count, shard, int(t), C.byref(gr), LOG_SCALE_MIN,
                                                   LOG_SCALE_MAX, OPACITY_LOGIT_MAX))

    def pack_params(self, lo, count, shard, out: DevBuf) -> None:
        self._check(self._lib().sc_splats_pack_range(self.ctx.handle, self.g.handle, lo, count, shard, out.cptr))

    def unpack_params(self, gathered: DevBuf, n_shards, shard) -> None:
        self._check(self._lib().sc_splats_unpack_shards(self.ctx.handle, self.g.handle, gathered.cptr, n_shards,
                                                        shard))

    def pack_moments(self, lo, count, shard, out: DevBuf) -> None:
        self._check(self._lib().sc_moments_pack_range(self.ctx.handle, self.mo.handle, lo, count, shard, out.cptr))

    def unpack_moments(self, gathered: DevBuf, n_shards, shard) -> None:
        self._check(self._lib().sc_moments_unpack_shards(self.ctx.handle, self.mo.handle, self.g.n, gathered.cptr,
                                                         n_shards, shard))

    def grad_acc(self) -> DevBuf:
        return self.acc

    def densify_prune(self, it, grad_count, do_prune, do_densify) -> None:
        from .adam_gpu import (DENSIFY_GRAD_THRESHOLD, PRUNE_OPACITY_LOGIT, SPLIT_SCALE_THRESHOLD, densify,
                               prune_low_opacity)
        if do_prune:
            prune_low_opacity(self.ctx, self.g, self.mo, self._acc, PRUNE_OPACITY_LOGIT)
        if do_densify:
            densify(self.ctx, self.g, self.mo, self._acc, grad_count, DENSIFY_GRAD_THRESHOLD, SPLIT_SCALE_THRESHOLD,
                    min(self.cfg.max_splats, self.g.capacity), it)
            self._acc.zero()

    def images(self) -> np.ndarray:
        return self.trainer.images()


def expected_shards(n: int, world: int) -> list[tuple[int, int]]:
    """(lo, count) of every rank; the chunks tile [0, n) exactly."""
    shard = shard_size(n, world)
    return [chunk_range(n, shard, r) for r in range(world)]
