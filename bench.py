"""Benchmark: fwd+bwd+Adam training iterations per second on the batched
1M-splat 1920x1080 workload (8 views per iteration).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one training iteration over n_views views: projection + SH,
binning + sorts, alpha-blend forward with fused MSE, blend backward, project
backward summed over views, densify statistic, Adam and constraints.  Inputs
(parameters, target images) live in HBM when the timed region starts; `e2e`
times the same step through the public API with the step's target images and
cameras copied from pinned host memory and the loss read back every step.

Rank 0 prints one JSON line.  `--impl reference` times the CPU restatement of
the reference path (the oracle, all host threads) on a bounded sample.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "fwd+bwd+Adam iters/s @1M splats 1080p: batched-BF16 vs plain FP32, same PSNR"
UNIT = "iters/s"


def profiled_traffic(kernel: str, views: int):
    """DRAM bytes per launch of a stage's dominant kernel from the committed ncu
    summaries (a line `traffic: kernel=<stage> views=<v> dram_bytes=<bytes>` of
    one capture), scaled from the captured views to `views`; None without one."""
    import re
    for f in sorted((ROOT / "profiles").glob("*.md")):
        m = re.search(r"traffic: kernel=(\w+) views=(\d+) dram_bytes=(\d+)", f.read_text())
        if m and m.group(1) == kernel:
            return int(int(m.group(3)) * views / int(m.group(2)))
    return None


# Arithmetic of one contributing (pixel, entry) pair, counted from the kernels'
# formulas (scalar FP operations, SFU included): the forward evaluates the
# Gaussian (offset, quadratic form, exp2, opacity clamp, the two cut tests: 11)
# and blends (T alpha, three colour FMAs, T update: 6); the backward evaluates
# the same 11, rebuilds T (1 - alpha, reciprocal, product: 3), forms T alpha,
# the colour gradient (3), dL/dC . c (3), dL/dalpha (2), the opacity term (1),
# its moments in y (3) and the running dot GS (1).  With two pixels per packed
# instruction and 32 lanes, a warp instruction does at most 64 of them.
PAIR_OPS = {"blend_fwd": 17, "blend_bwd": 29}


def profiled_instructions(kernel: str):
    """Warp instructions per contributing (pixel, entry) pair of a blend kernel
    from a committed ncu summary (a line `instructions: kernel=<stage> views=<v>
    warp_inst=<n> pixel_pairs=<p>`: one launch's smsp__inst_executed.sum and the
    pair counter of the same step), or None."""
    import re
    for f in sorted((ROOT / "profiles").glob("*.md")):
        for m in re.finditer(r"instructions: kernel=(\w+) views=(\d+) warp_inst=(\d+) pixel_pairs=(\d+)",
                             f.read_text()):
            if m.group(1) == kernel and int(m.group(4)) > 0:
                return int(m.group(3)) / int(m.group(4)), f.name
    return None


def issue_roofline(bw: dict) -> dict:
    """Instruction roofline of the two issue-bound blends: warp instructions
    per contributing (pixel, entry) pair (profiled) against PAIR_OPS / 64, the
    pair arithmetic alone at full lanes and full packing."""
    out = {}
    for kernel, key in (("blend_fwd", "fwd_pixel_pairs"), ("blend_bwd", "bwd_pixel_pairs")):
        prof = profiled_instructions(kernel)
        floor = PAIR_OPS[kernel] / 64.0
        e = {"pixel_pairs_per_step": bw.get(key), "min_warp_inst_per_pair": round(floor, 4)}
        if prof:
            e.update({"warp_inst_per_pair": round(prof[0], 4), "frac": round(floor / prof[0], 4),
                      "profile": prof[1]})
        out[kernel] = e
    return out


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clock / throttle sampling (100 ms period).  Started before the
    warm-up so samples exist for short timed regions; summary() keeps the
    samples taken inside [t0, t1] (host wall clock), or the nearest ones."""

    QUERY = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, device_index: int, raw_copy: str | None = None):
        self.dev = device_index
        self.proc = None
        self.raw_copy = raw_copy
        self.path = Path(tempfile.mkstemp(suffix=".csv")[1])

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def stop(self):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()
            self.proc = None

    def summary(self, t0: float, t1: float):
        import datetime
        try:
            text = self.path.read_text()
            if self.raw_copy:
                Path(self.raw_copy).parent.mkdir(exist_ok=True)
                Path(self.raw_copy).write_text(text)
        except Exception:
            text = ""
        rows = []
        for line in text.splitlines():
            r = [x.strip() for x in line.split(",")]
            if len(r) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(r[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                rows.append((ts, float(r[2]), float(r[3]), r[6:10]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        inside = [r for r in rows if t0 - 0.05 <= r[0] <= t1 + 0.05]
        if not inside:  # timed region shorter than the sampling period: nearest samples
            inside = sorted(rows, key=lambda r: min(abs(r[0] - t0), abs(r[0] - t1)))[:2]
        reasons = sorted({self.NAMES[k] for r in inside for k in range(4) if r[3][k] == "Active"})
        return {"sm_mhz": statistics.median([r[1] for r in inside]), "sm_max_mhz": max(r[2] for r in inside),
                "reasons": reasons, "samples": len(inside)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
        pg = dist
    return ws, rank, local, pg


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, x: float) -> float:
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


class _Cuda:
    """The few CUDA runtime calls the harness needs around the library, through
    cuda-python (cuda.bindings.runtime): events recorded on the library's
    stream, a device-wide synchronize, page-locked host buffers."""

    def __init__(self):
        self._rt = None

    @property
    def rt(self):
        if self._rt is None:
            from cuda.bindings import runtime
            self._rt = runtime
        return self._rt

    def check(self, err, what: str):
        if int(err) != 0:
            raise RuntimeError(f"{what}: CUDA error {int(err)}")

    def set_device(self, device: int):
        self.check(self.rt.cudaSetDevice(int(device))[0], "cudaSetDevice")

    def synchronize(self):
        self.check(self.rt.cudaDeviceSynchronize()[0], "cudaDeviceSynchronize")

    def Event(self):
        return _CudaEvent(self)

    def pinned_f32(self, n: int):
        return _Pinned(self, n)


class _CudaEvent:
    def __init__(self, cu: _Cuda):
        self.cu = cu
        err, self.ev = cu.rt.cudaEventCreate()
        cu.check(err, "cudaEventCreate")

    def record(self, stream: int):
        self.cu.check(self.cu.rt.cudaEventRecord(self.ev, self.cu.rt.cudaStream_t(int(stream)))[0], "cudaEventRecord")

    def elapsed_time(self, later: "_CudaEvent") -> float:
        err, ms = self.cu.rt.cudaEventElapsedTime(self.ev, later.ev)
        self.cu.check(err, "cudaEventElapsedTime")
        return float(ms)

    def __del__(self):
        try:
            self.cu.rt.cudaEventDestroy(self.ev)
        except Exception:
            pass


class _Pinned:
    """n float32 in page-locked host memory (cudaHostAlloc), viewed as numpy."""

    def __init__(self, cu: _Cuda, n: int):
        import ctypes
        self.cu, self.n = cu, int(n)
        err, self.ptr = cu.rt.cudaHostAlloc(4 * self.n, cu.rt.cudaHostAllocDefault)
        cu.check(err, "cudaHostAlloc")
        self.arr = np.ctypeslib.as_array((ctypes.c_float * self.n).from_address(int(self.ptr)))

    def numpy(self):
        return self.arr

    def data_ptr(self) -> int:
        return int(self.ptr)

    def numel(self) -> int:
        return self.n

    def __del__(self):
        try:
            self.arr = None
            self.cu.rt.cudaFreeHost(self.ptr)
        except Exception:
            pass


cu = _Cuda()


# ------------------------------------------------------------------ workload
def make_workload(args, rank, ctx):
    import nanotracer_b200 as nt
    from nanotracer_b200.scene import FOV_Y, orbit_views, perturbed, random_scene
    from nanotracer_b200.train import render_targets
    n, W, H, V = args.splats, args.width, args.height, args.views
    scene = random_scene(n, 0x5EED5EED + rank)
    tl = nt.TilingParams(W, H, args.tile_w, 8.0, tile_h_override=args.tile_h)
    cams_for = lambda step: [nt.CameraUniform.from_pose(*p, FOV_Y, W, H, n) for p in orbit_views(V, step)]
    target_scene = perturbed(scene)
    return scene, target_scene, tl, cams_for, render_targets


def render_views(ctx, g, cams, tl):
    """Float4 renders (V, H, W, 4) of a device splat store from cams through the
    stage API (64-bit reference-order binning); untimed, for the PSNR side data."""
    import nanotracer_b200 as nt
    from nanotracer_b200._lib import SC_KEYS_NATIVE64
    r, b = nt.Rasterizer(ctx), nt.TileBinner(ctx)
    V = len(cams)
    proj = r.alloc_projected(g, V)
    r.project(g, cams, proj)
    bins = b.bin(proj, g.n, tl, stride=g.capacity, n_views=V, key_mode=SC_KEYS_NATIVE64)
    img = r.alloc_image(tl.width, tl.height, V)
    r.composite(proj, bins, img, tl, stride=g.capacity, n_views=V)
    return img.readback(np.float32).reshape(V, tl.height, tl.width, 4)


def psnr_db(img4, tgt3) -> float:
    x = np.asarray(img4, np.float64)[..., :3]
    mse = float(np.mean((x - np.asarray(tgt3, np.float64)) ** 2))
    return round(10.0 * math.log10(1.0 / max(mse, 1e-30)), 4)


CROP = (928, 512, 64)  # x0, y0 and side of the 64x64 crop of view 0 (tile-aligned, image centre)


def crop_fp64(host_splats, cam, W, H):
    """The 64x64 crop of view 0 rendered by the oracle's FP64 instantiation:
    projection of every splat in FP64, means shifted into the crop, 64-bit
    (tile, depth) binning and blend of the crop's tiles.  A pixel's colour
    depends only on its offset from each mean, so this is the crop of the
    full FP64 render."""
    from oracle import oracle as O
    x0, y0, side = CROP
    n = len(host_splats)
    os_ = O.OSplats.from_buffer(host_splats)
    rec = O.project(os_, O.camera_from_struct(bytes(cam.c)), "f64")
    rec[:, 0] -= x0
    rec[:, 1] -= y0
    otl = O.tiling(side, side, 16, 16, 8.0)
    _, pay, ranges = O.bin64(rec, 1, otl, "f64")
    img, _, _ = O.composite(rec, pay, ranges.reshape(-1), otl, "f64")
    del n
    return img


def quality(ctx, g, cams, tl, tgt, fp64=True):
    """PSNR of a form's final parameters over the iteration's views, and on the
    64x64 crop of view 0 for the GPU render and the FP64 oracle's render of the
    same parameters (the "PSNR within 0.05 dB of the FP64 oracle" statement)."""
    img = render_views(ctx, g, cams, tl)
    out = {"psnr_views": psnr_db(img, tgt)}
    if fp64:
        x0, y0, side = CROP
        tc = tgt[0, y0:y0 + side, x0:x0 + side]
        gc = img[0, y0:y0 + side, x0:x0 + side]
        oc = crop_fp64(g.readback(), cams[0], tl.width, tl.height)
        out["crop_gpu"] = psnr_db(gc, tc)
        out["crop_fp64"] = psnr_db(oc, tc)
        out["crop_delta_db"] = round(out["crop_gpu"] - out["crop_fp64"], 4)
        out["crop_max_abs_err"] = float(np.abs(gc.astype(np.float64) - oc).max())
    return out


def timed_run(ctx, stream, tr, g, mo, acc, cams_seq, t):
    """Steps over cams_seq between CUDA events on the library stream; returns (ms, t, loss)."""
    e0 = cu.Event()
    e1 = cu.Event()
    cu.synchronize()
    e0.record(stream)
    loss = None
    for cams in cams_seq:
        t += 1
        loss = tr.step(g, mo, acc, cams, t)
    e1.record(stream)
    cu.synchronize()
    return e0.elapsed_time(e1), t, loss


def side_forms(ctx, stream, args, scene, tbuf, tgt0, cams0, tl, n_steps, main_form):
    """The metric's other forms on the same box, from the same start, untimed
    except for their own K steps: the batched form in the other precision, and
    the plain FP32 form (one view per iteration, the reference's train() loop,
    train.rs:155-250), whose iterations cycle through the same views with the
    view's target copied into place every iteration (inside its timed region).
    Every form's final parameters go through quality()."""
    import nanotracer_b200 as nt
    from nanotracer_b200.train import TrainConfig, Trainer
    V, K, W = args.views, args.steps, args.warmup
    out = {}
    other = "fp32" if main_form == "bf16" else "bf16"
    bf16 = other == "bf16"
    cfg = TrainConfig(n_views=V, width=args.width, height=args.height, tile_w=tl.tile_w, tile_h=tl.tile_h,
                      depth_max=8.0, exact_backward=True, use_graph=True, bf16=bf16, densify=False)
    g = nt.GpuSplatBuffer.upload(ctx, scene, bf16_rest=bf16)
    mo = nt.AdamMomentBuffers(ctx, g.capacity, bf16=bf16)
    acc = ctx.storage_buffer_zeroed("grad_acc", 4 * g.capacity)
    tr = Trainer(ctx, cfg)
    tr.set_targets(tbuf)
    t = 0
    _, t, _ = timed_run(ctx, stream, tr, g, mo, acc, [cams0] * (n_steps - K), t)
    ms, t, _ = timed_run(ctx, stream, tr, g, mo, acc, [cams0] * K, t)
    out["batched_" + other] = {"iters_s": round(K / (ms / 1e3), 3), "ms_per_iter": round(ms / K, 4),
                               "views_per_iter": V, "iters": t, **quality(ctx, g, cams0, tl, tgt0)}
    del tr
    # plain FP32: one view per iteration, V times as many iterations (the same views seen as often)
    P3 = args.width * args.height * 3 * 4
    cfg1 = TrainConfig(n_views=1, width=args.width, height=args.height, tile_w=tl.tile_w, tile_h=tl.tile_h,
                       depth_max=8.0, exact_backward=True, use_graph=True, bf16=False, densify=False)
    g1 = nt.GpuSplatBuffer.upload(ctx, scene)
    mo1 = nt.AdamMomentBuffers(ctx, g1.capacity)
    acc1 = ctx.storage_buffer_zeroed("grad_acc", 4 * g1.capacity)
    one = ctx.storage_buffer_zeroed("target_view", P3)
    tr1 = Trainer(ctx, cfg1)
    tr1.set_targets(one)

    def plain(iters, t):
        for j in range(iters):
            v = j % V
            one.copy_from(tbuf, P3, src_offset=v * P3)
            t += 1
            tr1.step(g1, mo1, acc1, [cams0[v]], t)
        return t

    t1 = plain(V * (n_steps - K), 0)
    cu.synchronize()
    e0, e1 = cu.Event(), cu.Event()
    e0.record(stream)
    t1 = plain(V * K, t1)
    e1.record(stream)
    cu.synchronize()
    ms1 = e0.elapsed_time(e1)
    out["plain_fp32"] = {"iters_s": round(V * K / (ms1 / 1e3), 3), "ms_per_iter": round(ms1 / (V * K), 4),
                         "views_per_iter": 1, "iters": t1, **quality(ctx, g1, cams0, tl, tgt0)}
    del tr1
    return out


def stage_bytes(N: int, V: int, P: int, K: int, items: int, bw: dict, bf16: bool, tiles: int,
                adam: bool = True) -> dict:
    """Algorithmic bytes per step of each stage: N splats, V views of P pixels,
    K (tile, splat) pairs, `items` two-level items, the blends' work counters
    `bw`; `adam` false for the split-views step, whose last stage writes the
    gradient rows only (Adam runs after the reduce-scatter)."""
    rest_b = 90 if bf16 else 180
    mom_b = 59 * 2 * (2 if bf16 else 4)
    fwd_list = bw.get("fwd_scanned", 0) * 8 + bw.get("fwd_blended", 0) * 48  # item words + blended records
    bwd_list = bw.get("bwd_scanned", 0) * 8 + bw.get("bwd_blended", 0) * 48
    tile_passes = max(1, math.ceil(max(1, (tiles - 1).bit_length()) / 8))
    return {
        # records, zeroed gradient records, depth key, id, item count
        "project": N * (56 + rest_b) + V * N * (48 + 48 + 4 + 4 + 4),
        # segmented onesweep over the 16-bit depth keys: a histogram read, then 2 passes
        # of 8-bit digits each reading and writing key + id
        "depth_sort": V * N * 4 + 2 * V * N * 16,
        "count_scan": V * N * (4 + 4 + 4) + V * N * 8,
        "emit": V * N * (4 + 16 + 4) + K * 8,
        "tile_sort": K * 4 + tile_passes * K * 16,
        "ranges": K * 4 + tiles * 8,
        # two-level binning: items (member mask | super tile, splat); the blends
        # read each tile's super-tile item list up to where its pixels saturate
        "item_emit": V * N * (4 + 16 + 4) + items * 8,
        "item_sort": items * 4 + items * 16,   # histogram read + one 9-bit pass
        "item_ranges": items * 4,
        "blend_fwd": fwd_list + V * P * (16 + 8),
        "blend_bwd": bwd_list + V * P * (16 + 8 + 12) + V * N * 48,
        # projection backward: per-view gradient records + geometry in, 59 f32 gradient
        # rows out; streaming Adam: rows, parameters, moments and statistic in and out
        "bwd_adam": (V * N * 48 + N * 44 + N * 236 +
                     ((N * 236 + N * 2 * (56 + rest_b) + N * 2 * mom_b + N * 8) if adam else 0)),
    }


def run_ours(args):
    ws, rank, local, pg = dist_setup()
    if (ws > 1 and args.parallel == "views") or args.view_path:
        return run_views(args, ws, rank, local, pg)

    import nanotracer_b200 as nt
    from nanotracer_b200.train import TrainConfig, Trainer
    ctx = nt.CudaCtx(local)
    cu.set_device(local)  # this process's events and host buffers on the library's device
    stream = ctx.stream
    scene, tscene, tl, cams_for, render_targets = make_workload(args, rank, ctx)
    V = args.views
    bf16 = args.form == "bf16"
    cfg = TrainConfig(n_views=V, width=args.width, height=args.height, tile_w=args.tile_w, tile_h=args.tile_h,
                      depth_max=8.0, exact_backward=True, use_graph=True, bf16=bf16, densify=False)
    # the iteration's V views (radius-4 orbit, elevation jitter) and their targets;
    # every step trains on them, so the loss and PSNR are meaningful
    cams0 = cams_for(0)
    tgt0 = render_targets(ctx, tscene, cams0, tl)
    tbuf = ctx.storage_buffer("targets", tgt0)
    tune = None
    if args.autotune:  # untimed: scratch copies of the scene, before the timed trainer exists
        from nanotracer_b200.autotune import autotune
        cfg, trials = autotune(ctx, scene, cams0, tbuf, cfg)
        tune = {"choice": f"{cfg.tile_w}x{cfg.tile_h} tiles, sort_mode {cfg.sort_mode}, blend batch "
                          f"{cfg.blend_batch or 'all threads'}, sort digits {cfg.sort_digit_bits or 'auto'}",
                "trial_ms": {t.label: (round(t.ms, 3) if t.ms is not None else t.error) for t in trials},
                "identical_images_per_tile_shape": all(
                    len({t.digest for t in trials if t.digest and (t.tile_w, t.tile_h) == s}) <= 1
                    for s in {(t.tile_w, t.tile_h) for t in trials})}
        tl = nt.TilingParams(args.width, args.height, cfg.tile_w, 8.0, tile_h_override=cfg.tile_h)
    g = nt.GpuSplatBuffer.upload(ctx, scene, bf16_rest=bf16)
    mo = nt.AdamMomentBuffers(ctx, g.capacity, bf16=bf16)
    acc = ctx.storage_buffer_zeroed("grad_acc", 4 * g.capacity)
    tr = Trainer(ctx, cfg)
    tr.set_targets(tbuf)
    clk = ClockSampler(local, raw_copy=os.environ.get("BENCH_CLOCKS_CSV")).start()
    t = 0
    for s in range(args.warmup):
        t += 1
        tr.step(g, mo, acc, cams0, t)
    cu.synchronize()
    barrier(pg)
    launches0 = ctx.launch_count
    e0 = cu.Event()
    e1 = cu.Event()
    cu.synchronize()
    w0 = time.time()
    e0.record(stream)
    for s in range(args.steps):
        t += 1
        loss = tr.step(g, mo, acc, cams0, t)
    e1.record(stream)
    cu.synchronize()
    w1 = time.time()
    clk.stop()
    barrier(pg)
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(pg, ms)
    launches = ctx.launch_count - launches0
    clocks = clk.summary(w0, w1)
    # stage times and blend work counters from further steps with the stage
    # events and counters on (outside the timed region, which runs without them)
    tr.set_profiling(True)
    for s in range(2):  # graph rebuild with profiling events
        t += 1
        tr.step(g, mo, acc, cams0, t)
    tr.set_profiling(True)  # reset the per-stage accumulators
    for s in range(min(args.steps, 10)):
        t += 1
        tr.step(g, mo, acc, cams0, t)
    st = tr.stats()
    # the blends' contributing (pixel, entry) pairs: two more steps with the pair counters on
    tr.set_profiling(2)
    for s in range(2):
        t += 1
        tr.step(g, mo, acc, cams0, t)
    tr.set_profiling(2)
    t += 1
    tr.step(g, mo, acc, cams0, t)
    for k in ("fwd_pixel_pairs", "bwd_pixel_pairs"):
        st["blend_work"][k] = tr.stats()["blend_work"][k]
    tr.set_profiling(True)
    n_steps = t
    forms = None
    if rank == 0 and ws == 1 and not args.no_forms:
        forms = {"batched_" + args.form: {"iters_s": round(args.steps / (ms / 1e3), 3),
                                          "ms_per_iter": round(ms / args.steps, 4), "views_per_iter": V,
                                          "iters": n_steps, **quality(ctx, g, cams0, tl, tgt0)}}

    # ---- e2e through the public API: pinned host targets + cameras in, loss out
    e2e = None
    if not args.no_e2e:
        # the step's targets come from pinned host memory: the trainer copies them
        # on a side stream every step, overlapped with the stages before the blend
        pinned = cu.pinned_f32(tgt0.size)
        pinned.numpy()[:] = tgt0.reshape(-1)
        tr.set_profiling(False)
        tr.set_host_targets(pinned.data_ptr(), keepalive=pinned)
        h2d = pinned.numel() * 4 + V * 96
        t += 1
        tr.step(g, mo, acc, cams0, t)  # re-capture the graph with the copy node (untimed)
        cu.synchronize()
        barrier(pg)
        t0 = time.perf_counter()
        f0 = cu.Event()
        f1 = cu.Event()
        f0.record(stream)
        for s in range(args.steps):
            t += 1
            tr.step(g, mo, acc, cams0, t)
        f1.record(stream)
        cu.synchronize()
        wall = time.perf_counter() - t0
        e2e_ms = max_over_ranks(pg, max(f0.elapsed_time(f1), wall * 1e3))
        e2e = {"value": ws * args.steps / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": 24}
    del tr

    # ---- roofline of the dominant stage
    stage = st["stage_ms"]
    dom = max(stage, key=stage.get)
    N = len(scene)
    bw = st.get("blend_work") or {}
    algo = stage_bytes(N, V, args.width * args.height, st["pairs"], st.get("items") or 0, bw, bf16,
                       V * tl.num_tiles())
    peaks = load_peaks()
    dom_ms = stage[dom]
    achieved = algo[dom] / (dom_ms / 1e3) / 1e9 if dom_ms > 0 else 0.0
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"],
                "unit": "GB/s", "frac": round(achieved / peaks["hbm_gbs"], 4),
                "traffic": profiled_traffic(dom, V),
                "peak_source": peaks["source"], "algorithmic_bytes": int(algo[dom]), "avg_ms": round(dom_ms, 4),
                "stage_ms": {k: round(v, 4) for k, v in stage.items()}, "blend_work": bw,
                "stage_frac_of_peak": {k: round(algo[k] / (v / 1e3) / 1e9 / peaks["hbm_gbs"], 4)
                                       for k, v in stage.items() if k in algo and v > 0},
                "issue": issue_roofline(bw)}

    if forms is not None:
        forms.update(side_forms(ctx, stream, args, scene, tbuf, tgt0, cams0, tl, n_steps, args.form))
        b, f, p = forms.get("batched_bf16"), forms.get("batched_fp32"), forms.get("plain_fp32")
        forms["bf16_over_fp32_batched"] = round(b["iters_s"] / f["iters_s"], 4) if b and f else None
        forms["bf16_batched_over_fp32_plain_iters"] = round(b["iters_s"] / p["iters_s"], 4) if b and p else None
        forms["bf16_batched_over_fp32_plain_views"] = \
            round(b["iters_s"] * V / p["iters_s"], 4) if b and p else None
        forms["psnr_delta_db_bf16_vs_fp32_batched"] = round(b["psnr_views"] - f["psnr_views"], 4) if b and f else None
        forms["crop"] = f"64x64 at ({CROP[0]}, {CROP[1]}) of view 0; FP64 = the oracle's double instantiation"

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args, scene, tl, cams0)

    if rank == 0:
        line = {
            "metric": METRIC, "value": ws * args.steps / (ms_max / 1e3), "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 blend/grad, bf16 SH-rest + Adam moments" if bf16 else "f32",
            "data": "synthetic seeded scene and targets (no dataset)",
            "config": {"workload": f"{N} splats, {V} views x {args.width}x{args.height} per iteration"
                                   f"{' per GPU (one scene per GPU)' if ws > 1 else ''}, "
                                   f"{cfg.tile_w}x{cfg.tile_h} tiles, exact transmittance backward, CUDA graph",
                       "form": "batched-" + ("bf16" if bf16 else "fp32"), "splats": N, "views_per_iter": V,
                       "width": args.width, "height": args.height, "pairs_per_iter": st["pairs"], "items_per_iter": st.get("items") or 0,
                       "l2": "inputs larger than L2 (params, item lists and images >> 126 MB)",
                       "parallelism": f"{ws} GPUs, one scene each (no exchange)" if ws > 1 else "single GPU"},
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": clocks, "loss": loss, "forms": forms,
        }
        if tune is not None:
            line["config"]["autotune"] = tune
        print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()


def run_precision(args):
    """The precision form, a side line beside the headline:
    3M splats, 4 views of 1920x1080 per iteration, SH-rest and Adam moments in
    BF16, blending and gradient sums in FP32, with and without the compensated
    cross-tile gradient sums.  Reports each variant's iterations/s, the
    per-image PSNR against the targets over the full views and, on the 64x64
    crop of each view, the GPU render's and the FP64 oracle's (same
    parameters), and the projected-gradient error on the crop against the
    FP64 oracle's adjoint (same records, bins, image and dL/dC; the crop's
    dL/dC only, so the oracle runs in seconds), plain and compensated."""

    import nanotracer_b200 as nt
    from nanotracer_b200._lib import SC_BWD_EXACT, SC_KEYS_NATIVE64
    from nanotracer_b200.train import TrainConfig, Trainer
    from oracle import oracle as O
    O.set_threads(O.max_threads())
    ctx = nt.CudaCtx(0)
    cu.set_device(0)  # this process's events and host buffers on the library's device
    stream = ctx.stream
    scene, tscene, tl, cams_for, render_targets = make_workload(args, 0, ctx)
    V, W, H = args.views, args.width, args.height
    cams0 = cams_for(0)
    tgt0 = render_targets(ctx, tscene, cams0, tl)
    tbuf = ctx.storage_buffer("targets", tgt0)
    out = {"metric": "precision form, 3M splats x 4 views of 1080p: iters/s and error against the FP64 oracle", "unit": UNIT,
           "config": {"workload": f"{len(scene)} splats, {V} views x {W}x{H} per iteration, BF16 SH-rest + Adam "
                                  f"moments, FP32 blend and gradient sums", "crop": f"64x64 at ({CROP[0]}, "
                                  f"{CROP[1]}) of every view"}}
    for comp in (False, True):
        cfg = TrainConfig(n_views=V, width=W, height=H, tile_w=args.tile_w, tile_h=args.tile_h, depth_max=8.0,
                          exact_backward=True, use_graph=True, bf16=True, densify=False, compensated_sums=comp)
        g = nt.GpuSplatBuffer.upload(ctx, scene, bf16_rest=True)
        mo = nt.AdamMomentBuffers(ctx, g.capacity, bf16=True)
        acc = ctx.storage_buffer_zeroed("grad_acc", 4 * g.capacity)
        tr = Trainer(ctx, cfg)
        tr.set_targets(tbuf)
        _, t, _ = timed_run(ctx, stream, tr, g, mo, acc, [cams0] * max(3, args.warmup), 0)
        ms, t, _ = timed_run(ctx, stream, tr, g, mo, acc, [cams0] * args.steps, t)
        del tr
        img = render_views(ctx, g, cams0, tl)
        x0, y0, side = CROP
        host = g.readback()
        per_view = []
        for v in range(V):
            tc = tgt0[v, y0:y0 + side, x0:x0 + side]
            oc = crop_fp64(host, cams0[v], W, H)
            gc = img[v, y0:y0 + side, x0:x0 + side]
            per_view.append({"psnr_full": psnr_db(img[v], tgt0[v]), "crop_gpu": psnr_db(gc, tc),
                             "crop_fp64": psnr_db(oc, tc), "crop_delta_db": round(psnr_db(gc, tc) - psnr_db(oc, tc), 4),
                             "crop_max_abs_err": float(np.abs(gc.astype(np.float64) - oc).max())})
        out["compensated" if comp else "plain"] = {"iters_s": round(args.steps / (ms / 1e3), 3),
                                                   "ms_per_iter": round(ms / args.steps, 4), "iters": t,
                                                   "views": per_view}
        del g, mo, acc
    # projected-gradient error on the crop of view 0: the records shifted into the crop, binned for it
    x0, y0, side = CROP
    pipe_g = nt.GpuSplatBuffer.upload(ctx, scene, bf16_rest=True)
    r = nt.Rasterizer(ctx)
    proj = r.alloc_projected(pipe_g, 1)
    r.project(pipe_g, [cams0[0]], proj)
    rec = proj.readback(np.float32).reshape(-1, 12)[:len(scene)].copy()
    rec[:, 0] -= x0
    rec[:, 1] -= y0
    ctl = nt.TilingParams(side, side, 16, 8.0)
    cproj = ctx.storage_buffer("crop_records", rec)
    bins = nt.TileBinner(ctx).bin(cproj, len(scene), ctl, key_mode=SC_KEYS_NATIVE64)
    cimg, caux = r.alloc_image(side, side), r.alloc_aux(side, side)
    r.composite(cproj, bins, cimg, ctl, stride=len(scene), aux=caux)
    gimg = cimg.readback(np.float32).reshape(side, side, 4)
    aux = caux.readback(np.uint32).reshape(side, side, 2)
    _, dl = O.mse(gimg, tgt0[0, y0:y0 + side, x0:x0 + side])
    dlb = ctx.storage_buffer("dl", dl.reshape(-1, 4).astype(np.float32))
    grads = {}
    for comp in (False, True):
        pg = ctx.storage_buffer_zeroed("pg", len(scene) * 48)
        r.composite_backward(cproj, bins, cimg, dlb, pg, ctl, stride=len(scene), mode=SC_BWD_EXACT, aux=caux,
                             compensated=comp)
        grads[comp] = pg.readback(np.float32).reshape(-1, 12)
    otl = O.tiling(side, side, 16, 16, 8.0)
    _, pay, ranges = O.bin64(rec, 1, otl)
    ref = O.composite_backward(rec.astype(np.float64), pay, ranges.reshape(-1), otl,
                               gimg.reshape(-1, 4).astype(np.float64), dl.astype(np.float64), SC_BWD_EXACT,
                               aux[..., 1].reshape(-1), aux[..., 0].view(np.float32).reshape(-1).astype(np.float64),
                               "f64")
    cols = [0, 1, 2, 4, 5, 6, 8, 9, 10]
    live = np.abs(ref[:, cols]).max(1) > 0
    for comp in (False, True):
        e = np.linalg.norm(grads[comp][live][:, cols] - ref[live][:, cols], axis=1) / \
            np.linalg.norm(ref[live][:, cols], axis=1)
        out["compensated" if comp else "plain"]["crop_grad_rel_err"] = {
            "splats": int(live.sum()), "median": float(np.median(e)), "p99": float(np.percentile(e, 99)),
            "max": float(e.max())}
    print(json.dumps(out))


def run_scenes(args):
    """An uneven batch of scenes, a side line beside the headline: 16
    independent scenes with splat counts log-uniform in [10k, 500k] and image
    sizes drawn from {512x512, 1024x768, 1920x1080}, one view each per
    iteration, stepped by one many-scene trainer (every stage one launch over
    all scenes, one CUDA graph), against the same scenes stepped by one
    single-scene trainer each, one after another.  Then the reference's
    densify / prune schedule per scene under a 6M total cap (densify by
    gradient threshold 2e-4, prune at opacity < 0.005) over a short run."""

    import nanotracer_b200 as nt
    from nanotracer_b200.scene import FOV_Y, orbit_views, perturbed, random_scene
    from nanotracer_b200.scenes import Scene, ScenesTrainer, densify_prune_scenes
    from nanotracer_b200.train import TrainConfig, Trainer, render_targets
    ctx = nt.CudaCtx(0)
    cu.set_device(0)  # this process's events and host buffers on the library's device
    stream = ctx.stream
    rng = np.random.default_rng(0x5CE7E5)
    sizes = [(512, 512), (1024, 768), (1920, 1080)]
    n_sc = 16
    counts = [int(x) for x in np.exp(rng.uniform(np.log(1e4), np.log(5e5), n_sc))]
    dims = [sizes[int(k)] for k in rng.integers(0, 3, n_sc)]
    maxW, maxH = max(d[0] for d in dims), max(d[1] for d in dims)
    scenes, cams, tgts = [], [], []
    for i, (n, (W, H)) in enumerate(zip(counts, dims)):
        s = random_scene(n, 0x5EED0000 + i)
        cam = nt.CameraUniform.from_pose(*orbit_views(8, 0)[i % 8], FOV_Y, W, H, n)
        tgts.append(render_targets(ctx, perturbed(s), [cam], nt.TilingParams(W, H, 16, 8.0))[0])
        scenes.append(s)
        cams.append(cam)
    # one trainer for all scenes
    st = ScenesTrainer(ctx, n_sc, maxW, maxH)
    for i in range(n_sc):
        st.set_scene(i, Scene.upload(ctx, scenes[i], tgts[i], capacity=2 * counts[i]))
    t = 0
    for _ in range(max(3, args.warmup)):
        t += 1
        st.step(cams, t)
    cu.synchronize()
    e0, e1 = cu.Event(), cu.Event()
    e0.record(stream)
    for _ in range(args.steps):
        t += 1
        losses = st.step(cams, t)
    e1.record(stream)
    cu.synchronize()
    ms_one = e0.elapsed_time(e1) / args.steps
    stats = st.stats()
    # the same scenes, one single-scene trainer each, stepped one after another
    singles = []
    for i in range(n_sc):
        W, H = dims[i]
        g = nt.GpuSplatBuffer.upload(ctx, scenes[i])
        mo = nt.AdamMomentBuffers(ctx, g.capacity)
        acc = ctx.storage_buffer_zeroed("acc", 4 * g.capacity)
        tr = Trainer(ctx, TrainConfig(n_views=1, width=W, height=H, depth_max=8.0))
        tr.set_targets(ctx.storage_buffer("t", np.ascontiguousarray(tgts[i], np.float32)))
        singles.append((tr, g, mo, acc))
    for k in range(max(3, args.warmup)):
        for i, (tr, g, mo, acc) in enumerate(singles):
            tr.step(g, mo, acc, [cams[i]], k + 1)
    cu.synchronize()
    e0.record(stream)
    for k in range(args.steps):
        for i, (tr, g, mo, acc) in enumerate(singles):
            tr.step(g, mo, acc, [cams[i]], k + 10)
    e1.record(stream)
    cu.synchronize()
    ms_sep = e0.elapsed_time(e1) / args.steps
    del singles
    # the densify / prune schedule (train.rs:259-362) per scene, 6M total cap
    sched = []
    w0 = time.perf_counter()
    for it in range(1, 201):
        t += 1
        st.step(cams, t)
        ev = densify_prune_scenes(st, it, grad_count=100, max_total=6_000_000, prune_every=100, prune_warmup=50,
                                  densify_every=100, densify_warmup=100)
        if any(ev.values()):
            sched.append({"iter": it, **ev, "total": sum(s.splats.n for s in st.scenes)})
    sched_s = time.perf_counter() - w0
    line = {"metric": "uneven batch: 16 scenes per iteration, one launch per stage", "unit": UNIT,
            "value": 1e3 / ms_one, "ms_per_iter": round(ms_one, 4), "steps": args.steps,
            "separate_trainers_ms_per_iter": round(ms_sep, 4),
            "speedup_over_separate_trainers": round(ms_sep / ms_one, 3),
            "config": {"scenes": n_sc, "splats": counts, "images": [f"{w}x{h}" for w, h in dims],
                       "total_splats": sum(counts), "tile_grid": f"{maxW}x{maxH}, 16x16 tiles"},
            "items_per_iter": stats["items"], "kernels_per_step": stats["kernels_per_step"],
            "loss_mean": float(np.mean(losses)),
            "densify_prune": {"iterations": 200, "wall_s": round(sched_s, 2), "events": sched,
                              "final_total": sum(s.splats.n for s in st.scenes)}}
    print(json.dumps(line))


def run_views(args, ws, rank, local, pg):
    """N ranks share one iteration of one scene: the iteration's views are split
    across the ranks (data-parallel views, one NCCL reduce-scatter of the
    gradients and one all-gather of the parameters per iteration).  Total work
    per iteration is fixed, so the scaling is strong."""

    import nanotracer_b200 as nt
    from nanotracer_b200.multiview import CudaCollectives, CudaViewBackend, ViewParallelTrainer, split_views
    from nanotracer_b200.nccl import NcclComm
    from nanotracer_b200.train import TrainConfig
    ctx = nt.CudaCtx(local)
    cu.set_device(local)  # this process's events and host buffers on the library's device
    # the data plane: NCCL through its C API on the library stream; its unique id
    # travels over TCP on the port after the launcher's (MASTER_PORT + 1)
    if ws > 1:
        comm = NcclComm(rank, ws, ctx.stream, os.environ.get("MASTER_ADDR", "127.0.0.1"),
                        int(os.environ.get("MASTER_PORT", "29500")) + 1)
    else:
        comm = NcclComm(0, 1, ctx.stream)
    scene, tscene, tl, cams_for, render_targets = make_workload(args, 0, ctx)  # one scene on every rank
    V = args.views
    bf16 = args.form == "bf16"
    cfg = TrainConfig(n_views=V, width=args.width, height=args.height, tile_w=args.tile_w, tile_h=args.tile_h,
                      depth_max=8.0, exact_backward=True, use_graph=True, bf16=bf16, densify=False)
    views = split_views(V, ws, rank)
    cams0 = cams_for(0)
    tgt_local = render_targets(ctx, tscene, [cams0[v] for v in views], tl)
    tgt_all = np.zeros((V,) + tgt_local.shape[1:], np.float32)
    tgt_all[views] = tgt_local
    be = CudaViewBackend(ctx, scene, cfg, tgt_all, views)
    tr = ViewParallelTrainer(be, V, CudaCollectives(ctx, comm))
    stream = ctx.stream
    cams_steps = [[cams_for(s)[v] for v in views] for s in range(args.warmup + args.steps)]
    clk = ClockSampler(local, raw_copy=os.environ.get("BENCH_CLOCKS_CSV")).start()
    t = 0
    for s in range(args.warmup):
        t += 1
        be.set_cameras(cams_steps[s])
        tr.step(t)
    cu.synchronize()
    barrier(pg)
    launches0 = ctx.launch_count
    e0 = cu.Event()
    e1 = cu.Event()
    w0 = time.time()
    e0.record(stream)
    for s in range(args.steps):
        t += 1
        be.set_cameras(cams_steps[args.warmup + s])
        loss = tr.step(t)
    e1.record(stream)
    cu.synchronize()
    w1 = time.time()
    clk.stop()
    barrier(pg)
    ms_max = max_over_ranks(pg, e0.elapsed_time(e1))
    launches = ctx.launch_count - launches0
    clocks = clk.summary(w0, w1)
    # stage times from further steps with the stage events on (every rank takes them)
    be.trainer.set_profiling(True)
    for s in range(2):  # graph rebuild with profiling events
        t += 1
        be.set_cameras(cams_steps[s])
        tr.step(t)
    be.trainer.set_profiling(True)  # reset the per-stage accumulators
    for s in range(min(args.steps, 10)):
        t += 1
        be.set_cameras(cams_steps[args.warmup + s])
        tr.step(t)
    st = be.trainer.stats()
    be.trainer.set_profiling(False)
    e2e = None
    if not args.no_e2e:
        # this rank's targets from page-locked host memory, copied by the trainer
        # every step on a side stream, view by view, beside the stages before the blend
        pinned = cu.pinned_f32(tgt_local.size)
        pinned.numpy()[:] = tgt_local.reshape(-1)
        be.trainer.set_host_targets(pinned.data_ptr(), keepalive=pinned)
        t += 1
        be.set_cameras(cams_steps[args.warmup])
        tr.step(t)  # re-capture the graph with the copy nodes (untimed; every rank takes it)
        cu.synchronize()
        barrier(pg)
        f0 = cu.Event()
        f1 = cu.Event()
        p0 = time.perf_counter()
        f0.record(stream)
        for s in range(args.steps):
            t += 1
            be.set_cameras(cams_steps[args.warmup + s])
            tr.step(t)
        f1.record(stream)
        cu.synchronize()
        wall = time.perf_counter() - p0
        e2e_ms = max_over_ranks(pg, max(f0.elapsed_time(f1), wall * 1e3))
        e2e = {"value": args.steps / (e2e_ms / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": int(pinned.numel() * 4 + len(views) * 96), "d2h_bytes_per_step": 24}
    stage = st["stage_ms"]
    dom = max(stage, key=stage.get)
    peaks = load_peaks()
    N, K, P, Vl = len(scene), st["pairs"], args.width * args.height, len(views)
    algo = stage_bytes(N, Vl, P, K, st.get("items") or 0, st.get("blend_work") or {}, bf16, Vl * tl.num_tiles(),
                       adam=False)
    ab = algo.get(dom)
    achieved = ab / (stage[dom] / 1e3) / 1e9 if ab and stage[dom] > 0 else None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": None if achieved is None else round(achieved, 1),
                "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": None if achieved is None else round(achieved / peaks["hbm_gbs"], 4), "traffic": None,
                "peak_source": peaks["source"], "algorithmic_bytes": ab, "avg_ms": round(stage[dom], 4),
                "stage_ms": {k: round(v, 4) for k, v in stage.items()}}
    if rank == 0:
        line = {
            "metric": METRIC, "value": args.steps / (ms_max / 1e3), "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32 blend/grad, bf16 SH-rest + Adam moments" if bf16 else "f32",
            "data": "synthetic seeded scene and targets (no dataset)",
            "config": {"workload": f"{N} splats, {V} views x {args.width}x{args.height} per iteration split over "
                                   f"{ws} GPUs, {args.tile_w}x{args.tile_h} tiles, exact transmittance backward",
                       "form": "batched-" + ("bf16" if bf16 else "fp32"), "splats": N, "views_per_iter": V,
                       "views_per_gpu": Vl, "width": args.width, "height": args.height,
                       "l2": "inputs larger than L2 (params, pair lists and images >> 126 MB)",
                       "parallelism": f"dp{ws} over views (NCCL reduce-scatter + all-gather through NCCL's C API "
                                      f"on the library stream, ZeRO-1 Adam)"},
            "roofline": roofline, "cpu_baseline": None, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": clocks, "loss": loss,
        }
        print(json.dumps(line))
    tr.close()
    del tr, be
    cu.synchronize()
    comm.close()
    if pg is not None:
        pg.destroy_process_group()


def cpu_baseline(args, scene, tl, cams):
    """The oracle (the CPU restatement of the reference path) on all host
    cores: one whole iteration of the workload (the V views' forward and
    backward over all splats, one Adam step) on the iteration's views."""
    from oracle import oracle as O
    from nanotracer_b200.train import BENCH_LRS
    threads = O.max_threads()
    O.set_threads(threads)
    n = len(scene)
    os_ = O.OSplats.from_buffer(scene)
    om, ov = O.OSplats.zeros(n), O.OSplats.zeros(n)
    acc = np.zeros(n, np.float32)
    ocams = [O.camera_from_struct(bytes(c.c)) for c in cams]
    tgt = np.zeros((len(cams), tl.height, tl.width, 3), np.float32)
    otl = O.tiling(tl.width, tl.height, tl.tile_w, tl.tile_h, tl.depth_max)
    t0 = time.perf_counter()
    O.train_step(os_, om, ov, acc, ocams, tgt, otl, 1, BENCH_LRS, 1)
    dt = time.perf_counter() - t0
    return {"value": 1.0 / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"one whole iteration ({len(cams)} views of {tl.width}x{tl.height}, {n} splats, "
                      f"fwd+bwd+Adam) in {dt:.2f} s"}


# The reference arm's bounded run: a few whole iterations (each one takes tens
# of seconds on the host cores), after fewer warm-up iterations than asked.
REF_MAX_STEPS = 3
REF_MAX_WARMUP = 1


def run_reference(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from nanotracer_b200.scene import FOV_Y, orbit_views, random_scene
    from oracle import oracle as O
    from nanotracer_b200.train import BENCH_LRS
    threads = O.max_threads()
    n, V, W, H = args.splats, args.views, args.width, args.height
    scene = random_scene(n, 0x5EED5EED)
    otl = O.tiling(W, H, args.tile_w, args.tile_h, 8.0)
    cams = [O.camera(*p, FOV_Y, W, H, n) for p in orbit_views(V, 0)]
    tgt = np.zeros((V, H, W, 3), np.float32)

    def fresh():
        return O.OSplats.from_buffer(scene), O.OSplats.zeros(n), O.OSplats.zeros(n), np.zeros(n, np.float32)

    # all host threads: whole V-view iterations
    O.set_threads(threads)
    os_, om, ov, acc = fresh()
    warm = min(args.warmup, REF_MAX_WARMUP)
    steps = max(1, min(args.steps, REF_MAX_STEPS))
    t = 0
    for _ in range(warm):
        t += 1
        O.train_step(os_, om, ov, acc, cams, tgt, otl, 1, BENCH_LRS, t)
    t0 = time.perf_counter()
    for _ in range(steps):
        t += 1
        O.train_step(os_, om, ov, acc, cams, tgt, otl, 1, BENCH_LRS, t)
    per_iter = (time.perf_counter() - t0) / steps
    v = 1.0 / per_iter
    # one thread: one view of the iteration (fwd+bwd over all splats, Adam over all parameters)
    O.set_threads(1)
    os1, om1, ov1, acc1 = fresh()
    s0 = time.perf_counter()
    O.train_step(os1, om1, ov1, acc1, cams[:1], tgt[:1], otl, 1, BENCH_LRS, 1)
    one_view = time.perf_counter() - s0
    O.set_threads(threads)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": steps,
            "warmup": warm, "ms_per_step": per_iter * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic seeded scene",
            "config": {"workload": f"{n} splats, {V} views x {W}x{H} per iteration"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{steps} whole iterations ({V} views, fwd+bwd over all {n} splats, one Adam "
                                       f"step each) after {warm} warm-up; asked for {args.steps} / {args.warmup}, "
                                       f"capped at {REF_MAX_STEPS} / {REF_MAX_WARMUP} to stay within minutes"},
            "cpu_1thread": {"seconds_per_view": round(one_view, 2), "cores": 1,
                            "iters_s_estimate": 1.0 / (one_view * V),
                            "sample": f"1 of the {V} views on one thread; iteration estimate = {V} x sample"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--splats", type=int, default=1_000_000)
    ap.add_argument("--views", type=int, default=8)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--tile-w", type=int, default=16)
    ap.add_argument("--tile-h", type=int, default=16)
    ap.add_argument("--form", default="bf16", choices=["bf16", "fp32"])
    ap.add_argument("--parallel", default="views", choices=["views", "scenes"],
                    help="N>1: split each iteration's views over the GPUs (strong), or one scene per GPU (weak)")
    ap.add_argument("--view-path", action="store_true", help="run the split-views path even on one GPU")
    ap.add_argument("--autotune", action="store_true",
                    help="time every tile shape x binning path first (untimed) and run the fastest")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the other forms' side runs (batched other precision, plain FP32) and their PSNR")
    ap.add_argument("--no-psnr", action="store_true", help=argparse.SUPPRESS)  # older name of --no-forms
    ap.add_argument("--workload", default="batched", choices=["batched", "precision", "scenes"],
                    help="precision: the precision-form side line (3M splats, 4 views, BF16, FP64-oracle errors); "
                         "scenes: the uneven-batch side line (16 uneven scenes in one launch per stage)")
    args = ap.parse_args()
    args.no_forms = args.no_forms or args.no_psnr
    if args.workload == "scenes":
        run_scenes(args)
        return
    if args.workload == "precision":
        if args.splats == 1_000_000 and args.views == 8:  # 3M splats x 4 views unless given
            args.splats, args.views = 3_000_000, 4
        run_precision(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        args.warmup = max(args.warmup, 3)
        run_ours(args)


if __name__ == "__main__":
    main()
