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
    relative (median) against FP64; with it every conic is within 1e-5, and
    the culling decisions (visible flags) equal the FP64 oracle's."""
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
    assert rel_on.max() <= 1e-5, rel_on.max()
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


def test_fp64_det_adjoint_differentiates_the_fp64_conic(ctx, oracle):
    """project_backward with the option recomputes the forward's FP64 conic:
    its geometric gradients (position, rotation, log-scale) of needles agree
    with the FP64 oracle's adjoint on the same projected gradients far better
    than the f32 adjoint does."""
    n, W, H = 4000, 1920, 1080
    s = needle_scene(n, 1.0, seed=5)
    cam = CameraUniform.from_pose(*orbit_pose(35.0), FOV_Y, W, H, n)
    rng = np.random.default_rng(11)
    pg = rng.normal(0.0, 1.0, (n, 12)).astype(np.float32)
    pg[:, [3, 7, 11]] = 0.0
    pg[:, 4:7] *= 1e3  # conic gradients carry the determinant's sensitivity
    os_ = oracle.OSplats.from_buffer(s)
    ref = oracle.project_backward(os_, pg, oracle.camera_from_struct(bytes(cam.c)), "f64")
    geo = slice(0, 10)

    def device(enabled):
        ctx.set_fp64_det(enabled)
        try:
            pipe = GpuPipe(ctx, s, cam, TilingParams(W, H, 16, 8.0))
            pipe.project()
            pgb = ctx.storage_buffer("pg", pg)
            grads = GradSplatBuffers(ctx, n)
            pipe.r.project_backward(pipe.g, pgb, cam, grads)
            return grads.readback(n).flat()
        finally:
            ctx.set_fp64_det(False)

    def rel(got):
        d = np.linalg.norm(got[:, geo] - ref[:, geo], axis=1)
        r = np.linalg.norm(ref[:, geo], axis=1)
        m = r > 0
        return d[m] / r[m]

    e_on, e_off = rel(device(True)), rel(device(False))
    assert np.median(e_on) <= 1e-4, np.median(e_on)
    assert np.percentile(e_on, 99) <= 1e-3, np.percentile(e_on, 99)
    assert np.median(e_off) >= 10 * np.median(e_on), (np.median(e_off), np.median(e_on))


def test_trainer_fp64_det_renders_what_the_fp64_projection_renders(ctx):
    """TrainConfig.fp64_det runs the same FP64 projection inside the captured
    step: its images equal, bit for bit, the stage path's with the context
    option on, and a step with needles moves every parameter to a finite value."""
    from nanotracer_b200._lib import SC_KEYS_NATIVE64
    from nanotracer_b200.train import render_targets
    from nanotracer_b200.scene import perturbed, orbit_views
    n, W, H, V = 2000, 256, 256, 2
    s = needle_scene(n, 0.3, seed=8)
    tl = TilingParams(W, H, 16, 8.0)
    cams = [CameraUniform.from_pose(*p, FOV_Y, W, H, n) for p in orbit_views(V, 0)]
    ctx.set_fp64_det(True)
    try:
        pipe = GpuPipe(ctx, s, cams, tl, key_mode=SC_KEYS_NATIVE64)
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
