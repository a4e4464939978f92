"""The precision form's FP64 step: near-degenerate (needle-like) splats get
their 2x2 projected-covariance determinant and inverse in FP64 when the
option is on (sc_ctx_set_fp64_det / TrainConfig.fp64_det), in the projection
and in its adjoint.  The reference forms det = s00 s11 - s01^2 in f32
(project_gaussians.wgsl:226-234), which cancellation ruins for needles.
Checked against the oracle's FP64 instantiation on the same f32 parameters."""
import math

import numpy as np
import pytest

from nanotracer_b200 import (AdamMomentBuffers, CameraUniform, GpuSplatBuffer, GradSplatBuffers, SplatBuffer,
                             TilingParams, TrainConfig, Trainer)
from nanotracer_b200.scene import FOV_Y, orbit_pose

from tests.util import GpuPipe

pytestmark = pytest.mark.gpu


def needle_scene(n, long_sigma, seed=3):
    """Splats with one axis of about long_sigma and two of 1e-4: their
    projections are lines whose f32 determinant cancels."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(-0.5, 0.5, (n, 3))
    scales = np.stack([np.full(n, math.log(long_sigma)), np.full(n, math.log(1e-4)), np.full(n, math.log(1e-4))], 1)
    scales = scales + rng.normal(0.0, 0.2, (n, 3))
    q = rng.normal(0.0, 1.0, (n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return SplatBuffer(pos, q, scales, rng.normal(0.0, 1.0, n), rng.normal(0.0, 0.3, (n, 3)),
                       rng.normal(0.0, 0.05, (n, 45)))


def _conic_rel(rec, ref):
    m = (rec[:, 7] == 1) & (ref[:, 7] == 1)
    c, r = rec[m, 4:7].astype(np.float64), ref[m, 4:7]
    return np.abs(c - r).max(1) / np.abs(r).max(1), m


def test_fp64_det_conic_of_needles_matches_the_fp64_oracle(ctx, oracle):
    """Without the option the f32 conic of 1080p needles is off by ~1e-3
    relative (median) against FP64; with it the conics of the splats that
    take the FP64 branch are within rounding of FP64 (median <= 1e-6) and
    those just above the branch's 2^-6 threshold keep at most 6 bits of
    cancellation (every conic within 1e-4), and the culling decisions
    (visible flags) equal the FP64 oracle's."""
    n, W, H = 4000, 1920, 1080
    s = needle_scene(n, 1.0)
    cam = CameraUniform.from_pose(*orbit_pose(20.0), FOV_Y, W, H, n)
    o = oracle.project(oracle.OSplats.from_buffer(s), oracle.camera_from_struct(bytes(cam.c)), "f64")
    tl = TilingParams(W, H, 16, 8.0)
    ctx.set_fp64_det(False)
    off = GpuPipe(ctx, s, cam, tl).project()[0]
    ctx.set_fp64_det(True)
    try:
        on = GpuPipe(ctx, s, cam, tl).project()[0]
    finally:
        ctx.set_fp64_det(False)
    rel_off, _ = _conic_rel(off, o)
    rel_on, m = _conic_rel(on, o)
    assert m.sum() > 0.9 * n
    assert np.array_equal(on[:, 7], o[:, 7].astype(np.float32))
    assert np.median(rel_off) > 1e-4, np.median(rel_off)   # the failure the option fixes
    assert np.median(rel_on) <= 1e-6, np.median(rel_on)
    assert rel_on.max() <= 1e-4, rel_on.max()
    print({"conic_rel_f32_median": float(np.median(rel_off)), "conic_rel_fp64_det_median": float(np.median(rel_on)),
           "conic_rel_fp64_det_max": float(rel_on.max())})
    # ordinary splats never take the FP64 branch: their records are unchanged
    from nanotracer_b200.scene import random_scene
    r = random_scene(2000, 4)
    a = GpuPipe(ctx, r, cam, tl).project()
    ctx.set_fp64_det(True)
    try:
        b = GpuPipe(ctx, r, cam, tl).project()
    finally:
        ctx.set_fp64_det(False)
    assert np.array_equal(a, b)


def test_fp64_det_adjoint_keeps_the_splats_the_forward_keeps(ctx, oracle):
    """Long needles (a long axis of about 20 against 1e-4) whose f32
    determinant cancels to <= 0: the f32 forward culls a share of them that
    the FP64 oracle keeps (project_gaussians.wgsl:226-234 culls det <= 0).
    With the option the forward keeps exactly the FP64 oracle's splats, and
    project_backward, which recomputes the same FP64 conic, gives a gradient
    to exactly those; without it forward and adjoint both cull them (the
    reference's f32 behaviour).  The adjoint's error against the FP64
    oracle's is printed for both; the rest of the adjoint chain stays f32
    (FP64 only for the 2x2 determinant and inverse), which dominates it."""
    n, W, H = 4000, 1920, 1080
    s = needle_scene(n, 20.0, seed=5)
    cam = CameraUniform.from_pose(*orbit_pose(35.0), FOV_Y, W, H, n)
    ocam = oracle.camera_from_struct(bytes(cam.c))
    os_ = oracle.OSplats.from_buffer(s)
    vis64 = oracle.project(os_, ocam, "f64")[:, 7] == 1
    rng = np.random.default_rng(11)
    pg = rng.normal(0.0, 1.0, (n, 12)).astype(np.float32)
    pg[:, [3, 7, 11]] = 0.0
    ref = oracle.project_backward(os_, pg, ocam, "f64")
    geo = slice(0, 10)

    def device(enabled):
        ctx.set_fp64_det(enabled)
        try:
            pipe = GpuPipe(ctx, s, cam, TilingParams(W, H, 16, 8.0))
            vis = pipe.project()[0][:, 7] == 1
            pgb = ctx.storage_buffer("pg", pg)
            grads = GradSplatBuffers(ctx, n)
            pipe.r.project_backward(pipe.g, pgb, cam, grads)
            return vis, grads.readback(n).flat()
        finally:
            ctx.set_fp64_det(False)

    vis_on, g_on = device(True)
    vis_off, g_off = device(False)
    assert (vis64 & ~vis_off).sum() > 100, "the scene does not exercise the f32 cancellation"
    assert np.array_equal(vis_on, vis64)
    assert np.array_equal(np.abs(g_on[:, geo]).sum(1) > 0, vis_on)
    assert np.array_equal(np.abs(g_off[:, geo]).sum(1) > 0, vis_off)
    assert np.array_equal(np.abs(ref[:, geo]).sum(1) > 0, vis64)

    def rel(got, m):
        d = np.linalg.norm(got[m][:, geo] - ref[m][:, geo], axis=1)
        return float(np.median(d / np.linalg.norm(ref[m][:, geo], axis=1)))

    print({"f32_culled_fp64_kept": int((vis64 & ~vis_off).sum()), "adjoint_rel_median_fp64_det": rel(g_on, vis_on),
           "adjoint_rel_median_f32_on_its_kept": rel(g_off, vis_off)})


def test_trainer_fp64_det_renders_what_the_fp64_projection_renders(ctx):
    """TrainConfig.fp64_det runs the same FP64 projection inside the captured
    step: its images equal, bit for bit, the stage path's with the context
    option on, and a step with needles moves every parameter to a finite value."""
    from nanotracer_b200._lib import SC_KEYS_REF32
    from nanotracer_b200.train import render_targets
    from nanotracer_b200.scene import perturbed, orbit_views
    n, W, H, V = 2000, 256, 256, 2
    s = needle_scene(n, 0.3, seed=8)
    tl = TilingParams(W, H, 16, 8.0)
    cams = [CameraUniform.from_pose(*p, FOV_Y, W, H, n) for p in orbit_views(V, 0)]
    ctx.set_fp64_det(True)
    try:
        pipe = GpuPipe(ctx, s, cams, tl, key_mode=SC_KEYS_REF32)
        pipe.project()
        pipe.bin()
        ref_img, _ = pipe.composite()
    finally:
        ctx.set_fp64_det(False)
    tgt = render_targets(ctx, perturbed(s), cams, tl)
    cfg = TrainConfig(n_views=V, width=W, height=H, depth_max=8.0, fp64_det=True)
    g = GpuSplatBuffer.upload(ctx, s)
    mo = AdamMomentBuffers(ctx, g.capacity)
    acc = ctx.storage_buffer_zeroed("acc", 4 * g.capacity)
    tr = Trainer(ctx, cfg)
    tr.set_targets(ctx.storage_buffer("targets", np.ascontiguousarray(tgt, np.float32)))
    loss = tr.step(g, mo, acc, cams, 1)
    assert np.isfinite(loss)
    assert np.array_equal(tr.images(), ref_img)
    assert np.all(np.isfinite(g.readback().flat()))


def _scene_with_backdrop(n, n_big, seed):
    """small-scene-like splats plus n_big large splats behind them whose
    footprints cover most of a 1080p view: their gradient totals add one term
    per tile over thousands of tiles."""
    from nanotracer_b200.scene import random_scene
    base = random_scene(n, seed).flat()
    rng = np.random.default_rng(seed + 1)
    big = base[:n_big].copy()
    big[:, 0:3] = rng.uniform(-0.3, 0.3, (n_big, 3))
    big[:, 7:10] = np.log(0.6) + rng.normal(0.0, 0.1, (n_big, 3))
    big[:, 10] = -2.0  # low opacity: the pixels behind stay unsaturated
    return SplatBuffer.from_flat(np.concatenate([base, big]).astype(np.float32))


def test_compensated_cross_tile_sums_against_the_fp64_oracle(ctx, oracle):
    """sc_composite_backward_ex(SC_BWD_FLAG_COMPENSATED) against the plain
    float atomics, both against the oracle's FP64 backward of the same records,
    bins, image and dL/dC: for splats whose totals add thousands of tile terms
    the compensated totals are closer to FP64, and everywhere they stay within
    the parity bound."""
    from nanotracer_b200._lib import SC_BWD_EXACT, SC_KEYS_NATIVE64
    from tests.util import check_pg_explained, margins
    W, H, n, n_big = 1920, 1080, 20000, 16
    s = _scene_with_backdrop(n, n_big, 17)
    cam = CameraUniform.from_pose(*orbit_pose(10.0), FOV_Y, W, H, n + n_big)
    tl = TilingParams(W, H, 16, 8.0)
    pipe = GpuPipe(ctx, s, cam, tl, key_mode=SC_KEYS_NATIVE64)
    rec = pipe.project()[0]
    _, pay, ranges = pipe.bin()
    img, aux = pipe.composite()
    rng = np.random.default_rng(4)
    dl = (rng.normal(size=(W * H, 4)) * 1e-6).astype(np.float32)
    dl[:, 3] = 0.0
    plain = pipe.backward(dl, SC_BWD_EXACT)[0].astype(np.float64)
    comp = pipe.backward(dl, SC_BWD_EXACT, compensated=True)[0].astype(np.float64)
    otl = oracle.tiling(W, H, 16, 16, 8.0)
    nc, tf = aux[0, ..., 1].reshape(-1), aux[0, ..., 0].view(np.float32).reshape(-1)
    ref = oracle.composite_backward(rec.astype(np.float64), pay, ranges.reshape(-1), otl,
                                    img[0].reshape(-1, 4).astype(np.float64), dl.astype(np.float64), SC_BWD_EXACT,
                                    nc, tf.astype(np.float64), "f64")
    _, absum = oracle.composite_backward(rec, pay, ranges.reshape(-1), otl, img[0].reshape(-1, 4), dl, SC_BWD_EXACT,
                                         nc, tf, want_abs=True)
    _, flags, _ = margins(oracle, rec, pay, ranges, otl, 1)
    cols = [0, 1, 2, 4, 5, 6, 8, 9, 10]
    big = np.arange(n, n + n_big)
    tiles = np.array([((rec[i, 3] * 2 / 16 + 1) ** 2) for i in big])
    rel = lambda g: np.abs(g[big][:, cols] - ref[big][:, cols]).max(1) / np.abs(ref[big][:, cols]).max(1)
    e_plain, e_comp = rel(plain), rel(comp)
    print({"tiles_per_big_splat_min": float(tiles.min()), "plain_rel_median": float(np.median(e_plain)),
           "comp_rel_median": float(np.median(e_comp)), "plain_rel_max": float(e_plain.max()),
           "comp_rel_max": float(e_comp.max())})
    assert tiles.min() > 1000
    assert np.median(e_comp) <= np.median(e_plain)
    assert e_comp.max() <= 1e-4
    check_pg_explained(comp.astype(np.float32), ref, absum, flags, label="compensated")
    check_pg_explained(plain.astype(np.float32), ref, absum, flags, label="plain")


def test_trainer_compensated_sums_step(ctx):
    """TrainConfig.compensated_sums: the same forward and loss, and the same
    first Adam step as the plain atomics except where a gradient's sign is
    within the sums' rounding (tests/util.py check_same_first_step)."""
    from nanotracer_b200.scene import orbit_views, perturbed, random_scene
    from nanotracer_b200.train import render_targets
    n, W, H, V = 20000, 256, 192, 2
    s = random_scene(n, 12)
    tl = TilingParams(W, H, 16, 8.0)
    cams = [CameraUniform.from_pose(*p, FOV_Y, W, H, n) for p in orbit_views(V, 0)]
    tgt = render_targets(ctx, perturbed(s), cams, tl)
    from tests.util import check_same_first_step
    out = []
    for comp in (False, True):
        g = GpuSplatBuffer.upload(ctx, s)
        mo = AdamMomentBuffers(ctx, g.capacity)
        acc = ctx.storage_buffer_zeroed("acc", 4 * g.capacity)
        cfg = TrainConfig(n_views=V, width=W, height=H, depth_max=8.0, compensated_sums=comp)
        tr = Trainer(ctx, cfg)
        tr.set_targets(ctx.storage_buffer("targets", np.ascontiguousarray(tgt, np.float32)))
        loss = tr.step(g, mo, acc, cams, 1)
        out.append((tr.images(), loss, g.readback().flat()))
    assert np.array_equal(out[0][0], out[1][0])
    assert abs(out[0][1] - out[1][1]) <= 1e-12 * out[0][1]
    print(check_same_first_step(out[0][2], out[1][2], cfg.lrs))
