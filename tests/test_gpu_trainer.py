"""The batched training step (sc_trainer): equivalence with the stage-by-stage
reference-shaped path, parity with the oracle's whole iteration, finite
differences through the device adjoint, graph replay, capacity growth."""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from nanotracer_b200 import (AdamMomentBuffers, CameraUniform, GpuSplatBuffer, GradSplatBuffers, SplatBuffer,
                             TilingParams, TrainConfig, Trainer)
from nanotracer_b200._lib import SC_BWD_EXACT, SC_BWD_REF, SC_KEYS_REF32
from nanotracer_b200.scene import FOV_Y, orbit_views, perturbed, random_scene
from nanotracer_b200.train import BENCH_LRS, render_targets

from tests.util import GpuPipe

pytestmark = pytest.mark.gpu
KATS = json.loads((Path(__file__).parent / "golden" / "reference_kats.json").read_text())


def _setup(ctx, n=3000, W=128, H=96, V=2, step=0, exact=True, graph=True, tile=(16, 16), bf16=False, seed=21):
    scene = random_scene(n, seed)
    tl = TilingParams(W, H, tile[0], 8.0, tile_h_override=tile[1])
    cams = [CameraUniform.from_pose(*p, FOV_Y, W, H, n) for p in orbit_views(V, step)]
    tgt = render_targets(ctx, perturbed(scene), cams, tl)
    cfg = TrainConfig(n_views=V, width=W, height=H, tile_w=tile[0], tile_h=tile[1], depth_max=8.0,
                      exact_backward=exact, use_graph=graph, bf16=bf16)
    return scene, tl, cams, tgt, cfg


def _run(ctx, scene, cams, tgt, cfg, steps=1, cap=0):
    g = GpuSplatBuffer.upload(ctx, scene, capacity=cap, bf16_rest=cfg.bf16)
    mo = AdamMomentBuffers(ctx, g.capacity, bf16=cfg.bf16)
    acc = ctx.storage_buffer_zeroed("acc", 4 * g.capacity)
    tr = Trainer(ctx, cfg)
    tb = ctx.storage_buffer("targets", np.ascontiguousarray(tgt, np.float32))
    tr.set_targets(tb)
    losses = [tr.step(g, mo, acc, cams, t) for t in range(1, steps + 1)]
    return tr, g, mo, acc, losses


@pytest.mark.parametrize("tile", [(16, 16), (8, 8), (32, 8)])
def test_trainer_images_equal_reference_order_binning(ctx, tile):
    """The trainer's 16-bit depth presort + stable tile sort reproduces the
    reference's 32-bit (tile << 16 | depth16) key order exactly, ties in the
    quantised depth going by splat index: its forward images equal, bit for
    bit, those of sc_bin(REF32) + sc_composite on the same records."""
    scene, tl, cams, tgt, cfg = _setup(ctx, V=3, tile=tile)
    pipe = GpuPipe(ctx, scene, cams, tl, key_mode=SC_KEYS_REF32)
    pipe.project()
    pipe.bin()
    ref_img, _ = pipe.composite()
    tr, *_ = _run(ctx, scene, cams, tgt, cfg)
    assert np.array_equal(tr.images(), ref_img)


def test_tile_culling_keeps_images_bit_identical_and_cuts_pairs(ctx):
    """Pairs whose alpha cannot reach 1/255 anywhere in the tile are dropped;
    the blend would skip them, so images are unchanged bit for bit."""
    scene, tl, cams, tgt, cfg = _setup(ctx, n=20000, W=256, H=192, V=2)
    cfg_off = TrainConfig(**{**cfg.__dict__, "tile_cull": False})
    tr_on, *_ = _run(ctx, scene, cams, tgt, cfg)
    tr_off, *_ = _run(ctx, scene, cams, tgt, cfg_off)
    assert np.array_equal(tr_on.images(), tr_off.images())
    assert tr_on.stats()["pairs"] < 0.95 * tr_off.stats()["pairs"]


@pytest.mark.parametrize("exact", [True, False])
def test_trainer_step_matches_oracle_iteration(ctx, oracle, exact):
    """One 2-view iteration (1500 splats, 96x64) checked stage by stage and
    through the captured step against the oracle (tests/parity.py)."""
    from tests.parity import iteration_parity
    scene, tl, cams, _, _ = _setup(ctx, n=1500, W=96, H=64, V=2, exact=exact)
    print(iteration_parity(ctx, oracle, scene, cams, tl, 1 if exact else 0, "small 2-view"))


def test_bf16_and_fp32_forms_within_0p05_db_of_the_fp64_oracle(ctx, oracle):
    """The precision target at a size the CPU finishes in seconds (2000
    splats, 2 views of 64x64): after 30 iterations from the same start, the
    PSNR of the BF16-storage form's images against the targets is within
    0.05 dB of the PSNR of the oracle's own run in f64 arithmetic, and so is
    the FP32 form's.  Images are each run's forward at the last iteration."""
    K, W, H = 30, 64, 64
    scene, tl, cams, tgt, cfg = _setup(ctx, n=2000, W=W, H=H, V=2, seed=9)
    t3 = np.asarray(tgt, np.float64).reshape(-1, 3)

    def psnr(img4):
        x = np.asarray(img4, np.float64).reshape(-1, 4)[:, :3]
        return 10.0 * math.log10(1.0 / np.mean((x - t3) ** 2))

    p = {}
    for name, bf16 in (("fp32", False), ("bf16", True)):
        tr, *_ = _run(ctx, scene, cams, tgt, TrainConfig(**{**cfg.__dict__, "bf16": bf16}), steps=K)
        p[name] = psnr(tr.images())
    os_ = oracle.OSplats.from_buffer(scene)
    om, ov = oracle.OSplats.zeros(len(scene)), oracle.OSplats.zeros(len(scene))
    oacc = np.zeros(len(scene), np.float32)
    ocams = [oracle.camera_from_struct(bytes(c.c)) for c in cams]
    otl = oracle.tiling(W, H, 16, 16, 8.0)
    for t in range(1, K + 1):
        _, oimgs = oracle.train_step(os_, om, ov, oacc, ocams, tgt, otl, 1, BENCH_LRS, t, sfx="f64",
                                     want_images=(t == K))
    p["fp64"] = psnr(oimgs)
    assert abs(p["bf16"] - p["fp64"]) <= 0.05, p
    assert abs(p["fp32"] - p["fp64"]) <= 0.05, p


def test_trainer_graph_replay_equals_eager(ctx):
    scene, tl, cams, tgt, cfg = _setup(ctx, n=2000)
    cfg_e = TrainConfig(**{**cfg.__dict__, "use_graph": False})
    _, g1, _, _, l1 = _run(ctx, scene, cams, tgt, cfg, steps=3)
    _, g2, _, _, l2 = _run(ctx, scene, cams, tgt, cfg_e, steps=3)
    # the backward's float atomics make the summation order (not the values) vary
    assert np.allclose(g1.readback().flat(), g2.readback().flat(), rtol=1e-5, atol=1e-7)
    assert np.allclose(l1, l2, rtol=1e-6)


def test_trainer_pair_capacity_growth(ctx):
    """A step that emits more pairs than the device capacity changes nothing,
    grows the buffers and runs again; the result equals a fresh run's."""
    small, tl, cams, tgt, cfg = _setup(ctx, n=200)
    big = random_scene(20000, 22)
    tgt_big = render_targets(ctx, perturbed(big), cams, tl)
    g = GpuSplatBuffer.upload(ctx, big)
    mo = AdamMomentBuffers(ctx, g.capacity)
    acc = ctx.storage_buffer_zeroed("acc", 4 * g.capacity)
    tr = Trainer(ctx, cfg)
    tr.set_targets(ctx.storage_buffer("t0", np.ascontiguousarray(tgt, np.float32)))
    gs = GpuSplatBuffer.upload(ctx, small)
    ms = AdamMomentBuffers(ctx, gs.capacity)
    accs = ctx.storage_buffer_zeroed("a", 4 * gs.capacity)
    tr.step(gs, ms, accs, cams, 1)  # sizes the pair buffers for the small scene
    small_pairs = tr.stats()["pairs"]
    tr.set_targets(ctx.storage_buffer("t1", np.ascontiguousarray(tgt_big, np.float32)))
    loss = tr.step(g, mo, acc, cams, 1)
    assert tr.stats()["pairs"] > 4 * small_pairs
    _, g2, _, _, l2 = _run(ctx, big, cams, tgt_big, cfg)
    assert abs(loss - l2[0]) <= 1e-9 * l2[0]
    assert np.allclose(g.readback().flat(), g2.readback().flat(), rtol=1e-5, atol=1e-7)


def test_finite_diff_through_device_adjoint(ctx):
    """backward_finite_diff.rs:173-246 on the device path (forward and analytic
    gradient both from the CUDA kernels), with the reference's tolerances."""
    k = KATS["finite_diff_matches_analytic"]
    sp, cm, t = k["splat"], k["camera"], k["tiling"]
    rest = np.zeros(45, np.float32)
    for i, v in sp["sh_rest"].items():
        rest[int(i)] = v
    base = SplatBuffer([sp["pos"]], [sp["rot"]], [sp["log_scale"]], [sp["opacity_logit"]], [sp["sh_dc"]], [rest])
    cam = CameraUniform.from_pose(cm["eye"], cm["target"], cm["up"], cm["fov_y"], cm["width"], cm["height"], 1)
    tl = TilingParams(cm["width"], cm["height"], t["tile_size"], t["depth_max"])

    def loss(s):
        p = GpuPipe(ctx, s, cam, tl)
        p.project()
        p.bin()
        img, _ = p.composite()
        return float(img[..., :3].astype(np.float64).sum())

    p = GpuPipe(ctx, base, cam, tl)
    p.project()
    p.bin()
    p.composite()
    p.backward(np.tile(np.array([1, 1, 1, 0], np.float32), (tl.width * tl.height, 1)), SC_BWD_REF)
    grads = GradSplatBuffers(ctx, 1)
    p.r.project_backward(p.g, p.pg, cam, grads)
    ga = grads.readback(1).flat()[0]
    eps = k["eps"]
    for name, col in {"sh_dc.r": 11, "opacity": 10, "sh_rest[0]": 14, "pos.x": 0, "log_scale.x": 7}.items():
        fp, fm = base.flat().copy(), base.flat().copy()
        fp[0, col] += eps
        fm[0, col] -= eps
        num = (loss(SplatBuffer.from_flat(fp)) - loss(SplatBuffer.from_flat(fm))) / (2 * eps)
        rel, ab = k["checks"][name]
        a = float(ga[col])
        assert abs(a - num) <= ab or abs(a - num) <= rel * (abs(a) + abs(num)), (name, a, num)


def test_bf16_storage_step_close_to_fp32(ctx):
    scene, tl, cams, tgt, cfg = _setup(ctx, n=3000)
    cfg16 = TrainConfig(**{**cfg.__dict__, "bf16": True})
    _, _, _, _, l32 = _run(ctx, scene, cams, tgt, cfg, steps=5)
    _, _, _, _, l16 = _run(ctx, scene, cams, tgt, cfg16, steps=5)
    assert abs(l16[0] - l32[0]) <= 2e-3 * l32[0]
    assert l16[-1] < l16[0] and l32[-1] < l32[0]


def test_host_targets_copied_beside_the_step_match_device_targets(ctx):
    import torch
    scene, tl, cams, tgt, cfg = _setup(ctx, n=2000, V=2)
    tr1, g1, _, _, l1 = _run(ctx, scene, cams, tgt, cfg, steps=2)
    g2 = GpuSplatBuffer.upload(ctx, scene)
    mo2 = AdamMomentBuffers(ctx, g2.capacity)
    acc2 = ctx.storage_buffer_zeroed("acc", 4 * g2.capacity)
    tr2 = Trainer(ctx, cfg)
    pinned = torch.empty(tgt.size, dtype=torch.float32, pin_memory=True)
    pinned.numpy()[:] = np.ascontiguousarray(tgt, np.float32).reshape(-1)
    tr2.set_host_targets(pinned.data_ptr(), keepalive=pinned)
    l2 = [tr2.step(g2, mo2, acc2, cams, t) for t in (1, 2)]
    assert np.array_equal(tr1.images(), tr2.images())
    assert np.allclose(l1, l2, rtol=1e-6)
    assert np.allclose(g1.readback().flat(), g2.readback().flat(), rtol=1e-5, atol=1e-7)
    # pageable memory is refused
    host = np.zeros(tgt.size, np.float32)
    with pytest.raises(Exception):
        tr2.set_host_targets(host.ctypes.data)


@pytest.mark.parametrize("tile", [(16, 16), (8, 8), (32, 8)])
def test_two_level_binning_equals_the_pair_sort(ctx, tile):
    """sort_mode 0/2 (super-tile item lists, each tile keeping the items whose
    member mask holds it) and sort_mode 1 (stable sort of the pairs) blend the
    same splats in the same order: the images and parameters after a step are
    identical, and the pair count summed from the masks equals the pair sort's."""
    scene, tl, cams, tgt, cfg = _setup(ctx, n=4000, V=3, tile=tile)
    assert cfg.sort_mode == 0
    tr2, g2, _, _, l2 = _run(ctx, scene, cams, tgt, cfg)        # default: two-level
    tr1, g1, _, _, l1 = _run(ctx, scene, cams, tgt, TrainConfig(**{**cfg.__dict__, "sort_mode": 1}))
    assert np.array_equal(tr1.images(), tr2.images())
    assert tr1.stats()["pairs"] == tr2.stats()["pairs"]
    assert tr2.stats()["items"] > 0 and tr1.stats()["items"] == 0
    assert np.allclose(l1, l2, rtol=1e-6)
    assert np.allclose(g1.readback().flat(), g2.readback().flat(), rtol=1e-5, atol=1e-7)


def test_full_size_binning_paths_agree(ctx):
    """The bench workload's sizes (1M splats, 8 views of 1920x1080, 16x16
    tiles), where the CPU oracle does not finish in seconds, checked through
    properties that hold at any size: the two-level binning and the stable
    pair sort blend the same splats in the same order (images bit for bit, the
    same pair count and loss), both equal the images of the reference's own
    binning (32-bit tile << 16 | depth16 keys, stable sort; 8 views x 8160
    tiles fit the 16 tile bits), and the blend work counters stay within each
    other and the pair count."""
    scene, tl, cams, tgt, cfg = _setup(ctx, n=1_000_000, W=1920, H=1080, V=8, seed=5)
    tr2, g2, mo2, acc2, l2 = _run(ctx, scene, cams, tgt, cfg)
    img2 = tr2.images()
    pairs2 = tr2.stats()["pairs"]
    tr1, _, _, _, l1 = _run(ctx, scene, cams, tgt, TrainConfig(**{**cfg.__dict__, "sort_mode": 1}))
    assert np.array_equal(tr1.images(), img2)
    assert tr1.stats()["pairs"] == pairs2 > 100_000_000
    assert np.allclose(l1, l2, rtol=1e-9)
    del tr1
    pipe = GpuPipe(ctx, scene, cams, tl, key_mode=SC_KEYS_REF32)
    pipe.project()
    pipe.bin()
    ref_img, _ = pipe.composite()
    assert np.array_equal(ref_img, img2)
    del pipe
    tr2.set_profiling(True)
    tr2.step(g2, mo2, acc2, cams, 2)
    st = tr2.stats()
    w = st["blend_work"]
    assert 0 < w["fwd_blended"] <= w["fwd_scanned"] <= st["items"] * 16
    assert 0 < w["bwd_blended"] <= w["bwd_scanned"] <= w["fwd_scanned"]
    assert w["bwd_blended"] <= w["fwd_blended"] <= st["pairs"]
    tr2.set_profiling(False)


def test_blend_work_counters_bound_each_other(ctx):
    """sc_trainer_blend_work while profiling: the forward blends only entries of
    the list positions it scans, the backward walks no further than the
    forward's last contributors, and neither touches more entries than there
    are (tile, splat) pairs."""
    scene, tl, cams, tgt, cfg = _setup(ctx, n=6000, V=3)
    g = GpuSplatBuffer.upload(ctx, scene)
    mo = AdamMomentBuffers(ctx, g.capacity)
    acc = ctx.storage_buffer_zeroed("acc", 4 * g.capacity)
    tr = Trainer(ctx, cfg)
    tr.set_targets(ctx.storage_buffer("targets", np.ascontiguousarray(tgt, np.float32)))
    tr.step(g, mo, acc, cams, 1)
    tr.set_profiling(True)
    for t in (2, 3):
        tr.step(g, mo, acc, cams, t)
    st = tr.stats()
    w = st["blend_work"]
    assert 0 < w["fwd_blended"] <= w["fwd_scanned"] <= st["items"] * 16
    assert 0 < w["bwd_blended"] <= w["bwd_scanned"] <= w["fwd_scanned"]
    assert w["bwd_blended"] <= w["fwd_blended"] <= st["pairs"]
    tr.set_profiling(False)


def test_pixel_pair_counters(ctx):
    """Profiling level 2 counts the blends' contributing (pixel, entry) pairs:
    with the exact backward the backward forms an adjoint for exactly the
    pairs the forward blended, the counts stay within the blended entries
    times the tile's pixels, level 1 leaves them at zero, and counting changes
    no image."""
    scene, tl, cams, tgt, cfg = _setup(ctx, n=6000, V=3)
    tr = Trainer(ctx, cfg)
    tr.set_targets(ctx.storage_buffer("targets", np.ascontiguousarray(tgt, np.float32)))
    out = []
    for level in (1, 2):
        g = GpuSplatBuffer.upload(ctx, scene)
        mo = AdamMomentBuffers(ctx, g.capacity)
        acc = ctx.storage_buffer_zeroed("acc", 4 * g.capacity)
        tr.set_profiling(level)
        tr.step(g, mo, acc, cams, 1)
        out.append((tr.stats()["blend_work"], tr.images()))
    (w1, img1), (w2, img2) = out
    assert w1["fwd_pixel_pairs"] == 0 and w1["bwd_pixel_pairs"] == 0
    assert np.array_equal(img1, img2)
    assert w2["fwd_blended"] == w1["fwd_blended"]
    assert 0 < w2["fwd_pixel_pairs"] == w2["bwd_pixel_pairs"]
    assert w2["fwd_pixel_pairs"] <= w2["fwd_blended"] * cfg.tile_w * cfg.tile_h
    tr.set_profiling(False)


def test_trainer_ragged_image_matches_oracle_iteration(ctx, oracle):
    """An image that is not a whole number of tiles (100x70 with 16x16 tiles:
    the last tile column and row hold 4 and 6 pixels): the iteration stage by
    stage and through the captured step against the oracle."""
    from tests.parity import iteration_parity
    scene, tl, cams, _, _ = _setup(ctx, n=1500, W=100, H=70, V=2)
    print(iteration_parity(ctx, oracle, scene, cams, tl, 1, "ragged 100x70"))


def test_trainer_step_with_every_splat_culled(ctx, oracle):
    """Every splat behind the camera: no items, empty lists, black images; the
    loss is the targets' mean square as in the oracle's iteration, and Adam's
    zero gradients leave every parameter where it was (the constraints
    renormalise the quaternions, a few ulp)."""
    n, W, H, V = 500, 64, 48, 2
    base = random_scene(n, 31).flat().copy()
    base[:, 0:3] = base[:, 0:3] * 0.1 + np.array([0.0, 0.0, 50.0], np.float32)  # far behind the orbit cameras
    scene = SplatBuffer.from_flat(base)
    tl = TilingParams(W, H, 16, 8.0)
    cams = [CameraUniform.from_pose((0.0, 0.0, -4.0), (0.0, 0.0, -10.0), (0.0, 1.0, 0.0), FOV_Y, W, H, n)] * V
    rng = np.random.default_rng(3)
    tgt = rng.uniform(0.0, 1.0, (V, H, W, 3)).astype(np.float32)
    cfg = TrainConfig(n_views=V, width=W, height=H, depth_max=8.0)
    tr, g, mo, acc, losses = _run(ctx, scene, cams, tgt, cfg)
    assert tr.stats()["items"] == 0 and tr.stats()["pairs"] == 0
    img = tr.images()
    assert np.all(img == 0.0)
    want = float(np.mean(tgt.astype(np.float64) ** 2))
    assert abs(losses[0] - want) <= 1e-6 * want, (losses[0], want)
    os_ = oracle.OSplats.from_buffer(scene)
    om, ov = oracle.OSplats.zeros(n), oracle.OSplats.zeros(n)
    ol, _ = oracle.train_step(os_, om, ov, np.zeros(n, np.float32), [oracle.camera_from_struct(bytes(c.c)) for c in cams],
                              tgt, oracle.tiling(W, H, 16, 16, 8.0), 1, BENCH_LRS, 1)
    assert abs(losses[0] - ol) <= 1e-6 * ol, (losses[0], ol)
    after, before = g.readback().flat(), scene.flat()
    rest = np.r_[0:3, 7:59]
    assert np.array_equal(after[:, rest], before[:, rest])
    assert np.allclose(after[:, 3:7], before[:, 3:7], rtol=0.0, atol=1e-6)


def test_trainer_culls_a_nonfinite_splat(ctx):
    """A splat whose position is NaN is culled (the projection's depth test
    rejects non-finite depths): the step renders what the same scene renders
    with that splat made transparent (an opacity logit of -30, below the 1/255
    cut everywhere, so it emits no item), bit for bit, and every other
    parameter stays finite."""
    scene, tl, cams, tgt, cfg = _setup(ctx, n=3000, V=2)
    f = scene.flat().copy()
    bad, away = f.copy(), f.copy()
    bad[17, 0] = np.nan
    away[17, 10] = -30.0
    tr_bad, g_bad, *_ = _run(ctx, SplatBuffer.from_flat(bad), cams, tgt, cfg)
    tr_away, *_ = _run(ctx, SplatBuffer.from_flat(away), cams, tgt, cfg)
    assert np.array_equal(tr_bad.images(), tr_away.images())
    out = g_bad.readback().flat()
    assert np.all(np.isfinite(np.delete(out, 17, axis=0)))


def test_trainer_step_with_no_splats(ctx):
    """An empty store (every splat pruned): the step runs, renders black and
    reports the targets' mean square as its loss."""
    W, H, V = 64, 48, 2
    scene = SplatBuffer.from_flat(np.zeros((0, 59), np.float32))
    cams = [CameraUniform.from_pose(*p, FOV_Y, W, H, 0) for p in orbit_views(V, 0)]
    tgt = np.random.default_rng(5).uniform(0.0, 1.0, (V, H, W, 3)).astype(np.float32)
    cfg = TrainConfig(n_views=V, width=W, height=H, depth_max=8.0)
    tr, g, mo, acc, losses = _run(ctx, scene, cams, tgt, cfg, cap=256)
    assert np.all(tr.images() == 0.0)
    want = float(np.mean(tgt.astype(np.float64) ** 2))
    assert abs(losses[0] - want) <= 1e-6 * want, (losses[0], want)
