"""CPU backend for ViewParallelTrainer built on the oracle, so the data-parallel
iteration (sharding arithmetic, reduce-scatter / all-gather sequence, shard
Adam, state gather before densify/prune) runs over gloo ranks without a GPU.
Test infrastructure only: the product backend is CudaViewBackend."""
from __future__ import annotations

import contextlib
import os

import numpy as np
import torch

from oracle import oracle as O

from nanotracer_b200.adam_gpu import DENSIFY_GRAD_THRESHOLD, PRUNE_OPACITY_LOGIT, SPLIT_SCALE_THRESHOLD
from nanotracer_b200.multiview import PARAM_ROWS, ViewParallelTrainer
from nanotracer_b200.scene import FOV_Y, orbit_views, perturbed, random_scene
from tests.torch_collectives import TorchCollectives

LRS = (1.6e-4, 1e-3, 5e-3, 0.05, 2.5e-3, 1.25e-4)
WIDTHS = (3, 4, 3, 1, 3, 45)  # parameter groups in row order


def problem(n=400, W=64, H=48, V=4, seed=7):
    """Scene, oracle cameras, tiling and float3 targets rendered by the oracle."""
    scene = random_scene(n, seed)
    tl = O.tiling(W, H, 16, 16, 8.0)
    cams = [O.camera(e, t, u, FOV_Y, W, H, n) for (e, t, u) in orbit_views(V, 0)]
    tgt_scene = O.OSplats.from_buffer(perturbed(scene))
    tg = []
    for c in cams:
        rec = O.project(tgt_scene, c)
        _, pay, ranges = O.bin_ref(rec, tl)
        img, _, _ = O.composite(rec, pay, ranges, tl)
        tg.append(img[..., :3])
    return scene, cams, tl, np.ascontiguousarray(np.stack(tg), np.float32)


def _rows(s: O.OSplats) -> np.ndarray:
    """(59, n) parameter rows of an oracle store."""
    return np.ascontiguousarray(s.flat().T)


def _set_rows(s: O.OSplats, rows: np.ndarray, lo: int, hi: int) -> None:
    """Copy columns lo:hi of (59, n) parameter rows into the store's per-group arrays."""
    r0 = 0
    for k, w in enumerate(WIDTHS):
        a = s.arrays[k][: s.n * w].reshape(s.n, w)
        a[lo:hi, :] = rows[r0:r0 + w, lo:hi].T
        r0 += w


class OracleViewBackend:
    def __init__(self, scene, cams, tl, targets, mode=1, capacity=None):
        self.device = torch.device("cpu")
        n = len(scene)
        cap = capacity or n
        self.s = O.OSplats.from_buffer(scene, cap)
        self.m, self.v = O.OSplats.zeros(n, cap), O.OSplats.zeros(n, cap)
        self.max_splats = 2 * n
        self.acc_np = np.zeros(max(cap, 1), np.float32)
        self.acc = torch.from_numpy(self.acc_np)
        self.cams, self.tl, self.targets, self.mode = cams, tl, targets, mode

    @property
    def n(self) -> int:
        return self.s.n

    def stream_context(self):
        return contextlib.nullcontext()

    def step_grads(self, views, loss_weight, n_shards, shard, grads) -> float:
        n = self.n
        g = np.zeros((n, PARAM_ROWS), np.float32)
        loss = 0.0
        for vi in views:
            rec = O.project(self.s, self.cams[vi])
            _, pay, ranges = O.bin_ref(rec, self.tl)
            img, ncon, tfin = O.composite(rec, pay, ranges, self.tl)
            lv, dl = O.mse(img, self.targets[vi], scale=loss_weight)
            loss += lv * loss_weight
            pg = O.composite_backward(rec, pay, ranges, self.tl, img, dl, self.mode, ncon, tfin)
            g += O.project_backward(self.s, pg, self.cams[vi])
        out = grads.numpy().reshape(n_shards, PARAM_ROWS, shard)
        out[:] = 0.0
        for q in range(n_shards):
            lo, hi = q * shard, min(n, (q + 1) * shard)
            if hi > lo:
                out[q, :, : hi - lo] = g[lo:hi].T
        return loss

    def adam_shard(self, chunk, lo, count, shard, t) -> None:
        if count == 0:
            return
        g = chunk.numpy().reshape(PARAM_ROWS, shard)[:, :count]
        self.acc_np[lo:lo + count] = O.accumulate_grad(np.ascontiguousarray(g[0:3].T), self.acc_np[lo:lo + count])
        p, m, v = _rows(self.s), _rows(self.m), _rows(self.v)
        r0 = 0
        for k, w in enumerate(WIDTHS):
            sl = slice(r0, r0 + w)
            np_, nm, nv = O.adam_step(p[sl, lo:lo + count], g[sl], m[sl, lo:lo + count], v[sl, lo:lo + count],
                                      LRS[k], t)
            p[sl, lo:lo + count], m[sl, lo:lo + count], v[sl, lo:lo + count] = np_, nm, nv
            r0 += w
        rot, sc, op = O.apply_constraints(p[3:7, lo:lo + count].T, p[7:10, lo:lo + count].T, p[10, lo:lo + count])
        p[3:7, lo:lo + count], p[7:10, lo:lo + count], p[10, lo:lo + count] = rot.T, sc.T, op
        _set_rows(self.s, p, lo, lo + count)
        _set_rows(self.m, m, lo, lo + count)
        _set_rows(self.v, v, lo, lo + count)

    def pack_params(self, lo, count, shard, out) -> None:
        o = out.numpy().reshape(PARAM_ROWS, shard)
        o[:] = 0.0
        o[:, :count] = _rows(self.s)[:, lo:lo + count]

    def unpack_params(self, gathered, n_shards, shard) -> None:
        g = gathered.numpy().reshape(n_shards, PARAM_ROWS, shard)
        rows = np.concatenate([g[q] for q in range(n_shards)], axis=1)[:, : self.n]
        _set_rows(self.s, rows, 0, self.n)

    def pack_moments(self, lo, count, shard, out) -> None:
        o = out.numpy().reshape(2, PARAM_ROWS, shard)
        o[:] = 0.0
        o[0, :, :count] = _rows(self.m)[:, lo:lo + count]
        o[1, :, :count] = _rows(self.v)[:, lo:lo + count]

    def unpack_moments(self, gathered, n_shards, shard) -> None:
        g = gathered.numpy().reshape(n_shards, 2, PARAM_ROWS, shard)
        for which, dst in ((0, self.m), (1, self.v)):
            rows = np.concatenate([g[q, which] for q in range(n_shards)], axis=1)[:, : self.n]
            _set_rows(dst, rows, 0, self.n)

    def grad_acc(self):
        return self.acc

    def densify_prune(self, it, grad_count, do_prune, do_densify) -> None:
        if do_prune:
            O.prune(self.s, self.m, self.v, self.acc_np, PRUNE_OPACITY_LOGIT)
        if do_densify:
            O.densify(self.s, self.m, self.v, self.acc_np, grad_count, DENSIFY_GRAD_THRESHOLD, SPLIT_SCALE_THRESHOLD,
                      self.max_splats, it)
            self.acc_np[:] = 0.0


def run_rank(rank, world, port, out_dir, steps, n, V, densify_at):
    """One gloo rank: `steps` split iterations, optional state gather + prune/densify."""
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        O.lib()
        O.set_threads(1)
        scene, cams, tl, tgt = problem(n=n, V=V)
        be = OracleViewBackend(scene, cams, tl, tgt, capacity=4 * n)
        tr = ViewParallelTrainer(be, V, TorchCollectives())
        losses = []
        grad_count = 0
        for t in range(1, steps + 1):
            losses.append(tr.step(t))
            grad_count += 1
            if densify_at and t == densify_at:
                tr.maybe_densify(t, grad_count, 0, 1, 0, 1)
                grad_count = 0
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), params=be.s.flat(), m=be.m.flat(), v=be.v.flat(),
                 acc=be.acc_np[: be.n], losses=np.array(losses), views=np.array(tr.views))
    finally:
        torch.distributed.destroy_process_group()


def run_rank_leaving(rank, world, port, out_dir):
    """Rank 1 leaves before the first collective; rank 0 must get an error, not hang."""
    import datetime
    import sys
    import time
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    O.lib()
    scene, cams, tl, tgt = problem(n=200, V=2)
    be = OracleViewBackend(scene, cams, tl, tgt)
    tr = ViewParallelTrainer(be, 2, TorchCollectives())
    if rank == 1:
        open(os.path.join(out_dir, "rank1.txt"), "w").write("left")
        sys.exit(0)  # between steps, with no collective in flight
    t0 = time.time()
    try:
        tr.step(1)
        outcome = "completed"
    except Exception as e:  # gloo reports the closed peer or the timeout
        outcome = "error:" + type(e).__name__
    open(os.path.join(out_dir, "rank0.txt"), "w").write(f"{outcome} {time.time() - t0:.1f}")
