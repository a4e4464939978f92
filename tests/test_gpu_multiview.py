"""Data-parallel views on the device: the gradient-only step, shard Adam and the
parameter pack/unpack, checked against the fused single-device step.

Two ranks are emulated on one GPU by running their steps one after the other
(no kernel waits on another rank); the reduce-scatter is the sum of the two
shard-major buffers.  The product exchange (NCCL through its C API on the
library stream, multiview.CudaCollectives) runs as a one-rank communicator."""
import ctypes as C
import os
import socket

import numpy as np
import pytest
import torch

from nanotracer_b200 import AdamMomentBuffers, CameraUniform, GpuSplatBuffer, TilingParams, TrainConfig, Trainer
from nanotracer_b200._lib import check, lib
from nanotracer_b200.adam_gpu import LOG_SCALE_MAX, LOG_SCALE_MIN, OPACITY_LOGIT_MAX, adam_groups
from nanotracer_b200.multiview import PARAM_ROWS, CudaViewBackend, ViewParallelTrainer, shard_size
from nanotracer_b200.raster import cameras_array
from nanotracer_b200.scene import FOV_Y, orbit_views, perturbed, random_scene
from nanotracer_b200.train import render_targets

pytestmark = pytest.mark.gpu


def _problem(ctx, n=2500, W=96, H=64, V=4, seed=11):
    scene = random_scene(n, seed)
    tl = TilingParams(W, H, 16, 8.0)
    cams = [CameraUniform.from_pose(*p, FOV_Y, W, H, n) for p in orbit_views(V, 0)]
    tgt = render_targets(ctx, perturbed(scene), cams, tl)
    cfg = TrainConfig(n_views=V, width=W, height=H, tile_w=16, tile_h=16, depth_max=8.0, exact_backward=True)
    return scene, cams, tgt, cfg


def _fused(ctx, scene, cams, tgt, cfg, steps=1):
    g = GpuSplatBuffer.upload(ctx, scene)
    mo = AdamMomentBuffers(ctx, g.capacity)
    acc = ctx.storage_buffer_zeroed("acc", 4 * g.capacity)
    tr = Trainer(ctx, cfg)
    tb = ctx.storage_buffer("t", np.ascontiguousarray(tgt, np.float32))
    tr.set_targets(tb)
    losses = [tr.step(g, mo, acc, cams, t) for t in range(1, steps + 1)]
    return g.readback().flat(), mo, acc.readback(np.float32, len(scene)), losses


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_emulated_two_rank_split_step_matches_fused(ctx):
    scene, cams, tgt, cfg = _problem(ctx)
    n, V, R = len(scene), len(cams), 2
    want, _, want_acc, want_loss = _fused(ctx, scene, cams, tgt, cfg)

    g = GpuSplatBuffer.upload(ctx, scene)
    mo = AdamMomentBuffers(ctx, g.capacity)
    acc = torch.zeros(g.capacity, dtype=torch.float32, device="cuda")
    shard = shard_size(n, R)
    grads = [torch.zeros(R * PARAM_ROWS * shard, dtype=torch.float32, device="cuda") for _ in range(R)]
    keep = []
    loss = 0.0
    for r, views in enumerate(([0, 1], [2, 3])):
        tr = Trainer(ctx, TrainConfig(**{**cfg.__dict__, "n_views": len(views)}))
        tb = ctx.storage_buffer("t", np.ascontiguousarray(tgt[views], np.float32))
        tr.set_targets(tb)
        keep += [tr, tb]
        lr = C.c_double()
        torch.cuda.synchronize()
        check(lib().sc_trainer_step_grads(tr.handle, g.handle, cameras_array([cams[v] for v in views]),
                                          C.c_float(1.0 / V), R, shard, _ptr(grads[r]), C.byref(lr)), ctx.handle)
        loss += lr.value
    assert abs(loss - want_loss[0]) <= 1e-6 * want_loss[0]
    total = (grads[0] + grads[1]).view(R, PARAM_ROWS * shard)
    # padding splats beyond n carry zero gradient
    pad = total.view(R, PARAM_ROWS, shard)[R - 1, :, n - (R - 1) * shard:]
    assert torch.count_nonzero(pad).item() == 0
    torch.cuda.synchronize()
    gathered = torch.zeros(R * PARAM_ROWS * shard, dtype=torch.float32, device="cuda")
    gr = adam_groups(cfg.lrs, cfg.beta1, cfg.beta2, cfg.eps)
    for r in range(R):
        lo, count = r * shard, min(shard, n - r * shard)
        check(lib().sc_adam_step_shard(ctx.handle, g.handle, mo.handle, _ptr(acc), _ptr(total[r]), lo, count, shard,
                                       1, C.byref(gr), LOG_SCALE_MIN, LOG_SCALE_MAX, OPACITY_LOGIT_MAX), ctx.handle)
        check(lib().sc_splats_pack_range(ctx.handle, g.handle, lo, count, shard,
                                         _ptr(gathered[r * PARAM_ROWS * shard:])), ctx.handle)
    ctx.synchronize()
    g2 = GpuSplatBuffer.upload(ctx, random_scene(n, 99))  # a different store, overwritten by the unpack
    check(lib().sc_splats_unpack_shards(ctx.handle, g2.handle, _ptr(gathered), R, shard), ctx.handle)
    got = g.readback().flat()
    # per-splat sums over two views then across the two halves: reassociation only
    assert np.mean(np.abs(got - want) <= 1e-6 + 1e-6 * np.abs(want)) > 0.995
    assert np.array_equal(g2.readback().flat(), got)
    assert np.allclose(acc[:n].cpu().numpy(), want_acc, rtol=1e-4, atol=1e-9 + 1e-5 * np.abs(want_acc).max())


def test_moments_pack_unpack_roundtrip(ctx):
    n, R = 1000, 3
    scene = random_scene(n, 5)
    g = GpuSplatBuffer.upload(ctx, scene)
    for bf16 in (False, True):
        mo = AdamMomentBuffers.upload_from_cpu(ctx, perturbed(scene), perturbed(perturbed(scene)), g.capacity, bf16)
        shard = shard_size(n, R)
        buf = torch.zeros(R * 2 * PARAM_ROWS * shard, dtype=torch.float32, device="cuda")
        for r in range(R):
            lo, count = r * shard, max(0, min(shard, n - r * shard))
            check(lib().sc_moments_pack_range(ctx.handle, mo.handle, lo, count, shard,
                                              _ptr(buf[r * 2 * PARAM_ROWS * shard:])), ctx.handle)
        mo2 = AdamMomentBuffers(ctx, g.capacity, bf16=bf16)
        ctx.synchronize()
        check(lib().sc_moments_unpack_shards(ctx.handle, mo2.handle, n, _ptr(buf), R, shard), ctx.handle)
        for x, y in zip(mo.download(n), mo2.download(n)):
            assert np.array_equal(x.flat(), y.flat())


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_view_parallel_trainer_one_rank_nccl_matches_fused(ctx):
    from nanotracer_b200.multiview import CudaCollectives
    from nanotracer_b200.nccl import NcclComm
    scene, cams, tgt, cfg = _problem(ctx, n=2000)
    want, _, _, want_loss = _fused(ctx, scene, cams, tgt, cfg, steps=2)
    comm = NcclComm(0, 1, ctx.stream, "127.0.0.1", _free_port())
    try:
        be = CudaViewBackend(ctx, scene, cfg, tgt, views=list(range(len(cams))))
        tr = ViewParallelTrainer(be, len(cams), CudaCollectives(ctx, comm))
        be.set_cameras([cams[v] for v in tr.views])
        losses = [tr.step(t) for t in (1, 2)]
        got = be.g.readback().flat()
        tr.gather_state()  # one rank: gathers its own chunk back in place
        assert np.array_equal(be.g.readback().flat(), got)
        tr.close()
    finally:
        comm.close()
    assert np.allclose(losses, want_loss, rtol=1e-6)
    assert np.mean(np.abs(got - want) <= 1e-6 + 1e-6 * np.abs(want)) > 0.995
