"""The SSIM and combined losses on the device (loss.rs:22-410) against the
oracle's restatement, and the trainer with an SSIM term against the oracle's
whole iteration."""
import ctypes as C

import numpy as np
import pytest

from nanotracer_b200._lib import check, lib, sc_tiling

from tests.test_gpu_trainer import _run, _setup

pytestmark = pytest.mark.gpu


def _tiling(w, h):
    t = sc_tiling()
    t.width, t.height, t.tile_w, t.tile_h, t.depth_max = w, h, 16, 16, 8.0
    return t


def _images(w, h, V, seed):
    rng = np.random.default_rng(seed)
    # smooth-ish content plus noise, values in [0, 1.2] like rendered radiance
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float32)
    base = 0.5 + 0.3 * np.sin(xx[None, ..., None] * 0.3 + np.arange(3) + np.arange(V)[:, None, None, None])
    pred = np.clip(base + 0.1 * rng.standard_normal((V, h, w, 3)), 0, 1.2).astype(np.float32)
    tgt = np.clip(base * 0.9 + 0.05 + 0.1 * rng.standard_normal((V, h, w, 3)), 0, 1.2).astype(np.float32)
    pred4 = np.concatenate([pred, rng.random((V, h, w, 1)).astype(np.float32)], axis=-1)
    return pred4, tgt


def _device_loss(ctx, fn, pred4, tgt, *args):
    V, h, w, _ = pred4.shape
    dp = ctx.storage_buffer("pred", pred4)
    dt = ctx.storage_buffer("tgt", tgt)
    dl = ctx.storage_buffer_zeroed("dl", pred4.nbytes)
    nl = 3 if fn == "sc_combined_loss_grad" else 1
    lo = ctx.storage_buffer_zeroed("loss", 8 * nl * V)
    t = _tiling(w, h)
    check(getattr(lib(), fn)(ctx.handle, dp.cptr, dt.cptr, V, C.byref(t), *args, dl.cptr, lo.cptr), ctx.handle)
    return lo.readback(np.float64).reshape(V, nl), dl.readback(np.float32).reshape(V, h, w, 4)


@pytest.mark.parametrize("w,h,V", [(64, 48, 1), (37, 23, 2), (8, 8, 1), (6, 6, 1), (200, 130, 1)])
def test_ssim_matches_oracle(ctx, oracle, w, h, V):
    pred4, tgt = _images(w, h, V, seed=w * h + V)
    loss, dl = _device_loss(ctx, "sc_ssim_loss_grad", pred4, tgt, C.c_float(1.0))
    for v in range(V):
        ol, odl = oracle.ssim(pred4[v], tgt[v], w, h)
        odl = odl.reshape(h, w, 4)
        assert abs(loss[v, 0] - ol) <= 1e-6 + 1e-5 * abs(ol)
        # forward arithmetic is the reference's; the transposed blur sums in another order
        scale = np.abs(odl).max()
        assert np.allclose(dl[v], odl, rtol=1e-4, atol=1e-5 * scale)
        assert np.all(dl[v][..., 3] == 0)


def test_ssim_gradient_against_fp64_oracle(ctx, oracle):
    w, h = 40, 30
    pred4, tgt = _images(w, h, 1, seed=3)
    _, dl = _device_loss(ctx, "sc_ssim_loss_grad", pred4, tgt, C.c_float(1.0))
    _, odl = oracle.ssim(pred4[0].astype(np.float64), tgt[0], w, h, sfx="f64")
    odl = odl.reshape(h, w, 4)
    assert np.allclose(dl[0], odl, rtol=1e-3, atol=1e-4 * np.abs(odl).max())


def test_ssim_identical_images_have_zero_loss(ctx):
    w, h = 32, 24
    pred4, _ = _images(w, h, 1, seed=9)
    loss, dl = _device_loss(ctx, "sc_ssim_loss_grad", pred4, np.ascontiguousarray(pred4[..., :3]), C.c_float(1.0))
    assert abs(loss[0, 0]) < 1e-5
    assert np.abs(dl).max() < 1e-5


@pytest.mark.parametrize("lam", [0.0, 0.2, 1.0])
def test_combined_loss_matches_oracle(ctx, oracle, lam):
    w, h, V = 48, 40, 2
    pred4, tgt = _images(w, h, V, seed=11)
    scale = 0.5
    parts, dl = _device_loss(ctx, "sc_combined_loss_grad", pred4, tgt, C.c_float(lam), C.c_float(scale))
    for v in range(V):
        total, m, s, odl = oracle.combined(pred4[v], tgt[v], w, h, lam, scale)
        odl = odl.reshape(h, w, 4)
        assert np.allclose(parts[v], [total, m, s], rtol=1e-5, atol=1e-7)
        assert np.allclose(dl[v], odl, rtol=1e-4, atol=1e-5 * np.abs(odl).max())
    if lam == 0.0:  # the pure MSE path, bit for bit
        _, dlm = _device_loss(ctx, "sc_mse_loss_grad", pred4, tgt, C.c_float(scale))
        assert np.array_equal(dl, dlm)


def test_ssim_rejects_tiny_images(ctx):
    pred4, tgt = _images(5, 8, 1, seed=1)
    with pytest.raises(Exception):
        _device_loss(ctx, "sc_ssim_loss_grad", pred4, tgt, C.c_float(1.0))


def test_trainer_with_ssim_term_matches_oracle_iteration(ctx, oracle):
    from nanotracer_b200.train import BENCH_LRS, TrainConfig
    lam = 0.2
    scene, tl, cams, tgt, cfg = _setup(ctx, n=1500, W=96, H=64, V=2, exact=True)
    cfg = TrainConfig(**{**cfg.__dict__, "ssim_lambda": lam})
    tr, g, mo, acc, losses = _run(ctx, scene, cams, tgt, cfg)
    os_ = oracle.OSplats.from_buffer(scene)
    om, ov = oracle.OSplats.zeros(len(scene)), oracle.OSplats.zeros(len(scene))
    oacc = np.zeros(len(scene), np.float32)
    ocams = [oracle.camera_from_struct(bytes(c.c)) for c in cams]
    oloss, _ = oracle.train_step(os_, om, ov, oacc, ocams, tgt, oracle.tiling(96, 64, 16, 16, 8.0), 1, BENCH_LRS, 1,
                                 ssim_lambda=lam)
    assert abs(losses[0] - oloss) <= 1e-5 * oloss
    got, want = g.readback().flat(), os_.flat()
    assert np.mean(np.abs(got - want) <= 1e-6 + 1e-6 * np.abs(want)) > 0.995
