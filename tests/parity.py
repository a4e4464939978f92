"""One training iteration checked against the oracle stage by stage, on
shared inputs, and through the captured training step (sc_trainer).

  projection   the oracle's f32 projection of the same parameters: same
               visibility, radius within 1 (the ceil of a rounded sqrt), the
               other fields within stated tolerances;
  bins         32-bit keys (tile << 16 | depth16), splat order and tile
               ranges from the GPU's records, bit-exact against the oracle's
               restatement of the reference's binning (stable key sort);
  image        within 1e-4 per pixel of the oracle's blend of the same
               records, every exception a pixel whose walk passes within a
               stated relative margin of a blend threshold (at most 0.1 %);
  gradients    projected gradients within 1e-3 relative plus 1e-4 of the sum
               of the terms' magnitudes (the rounding scale of a cancelling
               sum), the exceptions the near-threshold pixels' splats;
               parameter gradients per group within 1e-3 relative;
  trainer      images equal to the stage path's bit for bit, loss within
               1e-5, and the parameters after one Adam step equal to the
               oracle's Adam + constraints on the oracle's gradients, except
               groups whose gradient sign the tolerance leaves open.
"""
from __future__ import annotations

import time

import numpy as np

from nanotracer_b200 import AdamMomentBuffers, GpuSplatBuffer, GradSplatBuffers, TilingParams, TrainConfig, Trainer
from nanotracer_b200._lib import SC_KEYS_REF32
from nanotracer_b200.scene import perturbed
from nanotracer_b200.train import BENCH_LRS, render_targets

from tests.util import (GRAD_ABS_REL, GpuPipe, adam_first_step, check_image_explained, check_param_grads,
                        check_pg_explained, check_post_adam, margins)


def projection_report(g, o):
    """GPU records (n, 12) against the oracle's f32 projection of the same parameters."""
    same_vis = g[:, 7] == o[:, 7]
    m = same_vis & (o[:, 7] == 1)
    r = {"visible": int((o[:, 7] == 1).sum()), "visibility_mismatch": int((~same_vis).sum()),
         "radius_off_by_1": int((g[m, 3] != o[m, 3]).sum())}
    assert (~same_vis).sum() <= max(2, 1e-5 * len(g)), r
    if m.any():
        assert np.abs(g[m, 3] - o[m, 3]).max() <= 1.0, r
        assert (g[m, 3] != o[m, 3]).mean() <= 1e-3, r
        assert np.abs(g[m, 0:2] - o[m, 0:2]).max() < 2e-3, r
        assert np.allclose(g[m, 2], o[m, 2], rtol=2e-6), r
        conic_rel = np.abs(g[m, 4:7] - o[m, 4:7]).max(1) / np.abs(o[m, 4:7]).max(1)
        r["conic_rel_max"] = float(conic_rel.max())
        assert conic_rel.max() < 1e-4, r
        assert np.abs(g[m, 8:11] - o[m, 8:11]).max() < 1e-5, r
        assert np.abs(g[m, 11] - o[m, 11]).max() < 1e-6, r
    assert np.all(g[g[:, 7] == 0] == 0)
    return r


def iteration_parity(ctx, oracle, scene, cams, tl: TilingParams, mode: int, label: str, trainer=True) -> dict:
    n, V, W, H = len(scene), len(cams), tl.width, tl.height
    t0 = time.time()
    otl = oracle.tiling(W, H, tl.tile_w, tl.tile_h, tl.depth_max)
    ocams = [oracle.camera_from_struct(bytes(c.c)) for c in cams]
    os_ = oracle.OSplats.from_buffer(scene)
    report = {"config": label, "mode": mode}

    pipe = GpuPipe(ctx, scene, cams, tl, key_mode=SC_KEYS_REF32)
    rec = pipe.project()  # (V, n, 12)
    report["projection"] = [projection_report(rec[v], oracle.project(os_, ocams[v])) for v in range(V)]

    keys, pay, ranges = pipe.bin()
    ok, op, orr = oracle.bin_ref_views(rec.reshape(-1, 12), V, otl)
    report["pairs"] = int(len(ok))
    assert len(keys) == len(ok) and np.array_equal(keys, ok) and np.array_equal(pay, op)
    assert np.array_equal(ranges, orr)
    T = len(orr) // V

    img, aux = pipe.composite()
    tgt = np.asarray(render_targets(ctx, perturbed(scene), cams, tl), np.float32).reshape(V, H, W, 3)
    dl = np.zeros((V, H * W, 4), np.float32)
    flags_bwd = np.zeros(n, bool)  # splats whose gradient may differ given the same forward
    flags_fwd = np.zeros(n, bool)  # ... given each side's own forward
    per_view = []
    loss = 0.0
    for v in range(V):
        rv = ranges[v * T:(v + 1) * T].reshape(-1)
        oimg, _, _ = oracle.composite(rec[v], pay, rv, otl)
        margin, fb, ff = margins(oracle, rec[v], pay, rv, otl, mode)
        flags_bwd |= fb
        flags_fwd |= ff
        s = {"image": check_image_explained(img[v], oimg, margin, label=f"{label} view {v}")}
        lv, dlv = oracle.mse(img[v], tgt[v], 1.0 / V)
        loss += lv / V
        dl[v] = dlv.reshape(-1, 4)
        per_view.append(s)
    gpg = pipe.backward(dl.reshape(-1, 4), mode)  # (V, n, 12)
    grads = GradSplatBuffers(ctx, n)
    alt = np.zeros((n, 59), np.float64)  # the oracle's adjoint of the GPU's projected gradients
    # the absolute term of the projected-gradient bound carried to the opacity
    # logit (dsigma * s (1 - s)) and the SH coefficients (dcolor * basis, |basis| <= 1.1)
    unc = np.zeros((n, 59), np.float64)
    sig = 1.0 / (1.0 + np.exp(-scene.flat()[:, 10].astype(np.float64)))
    for v in range(V):
        rv = ranges[v * T:(v + 1) * T].reshape(-1)
        opg, absum = oracle.composite_backward(rec[v], pay, rv, otl, img[v].reshape(-1, 4), dl[v], mode,
                                               aux[v, ..., 1].reshape(-1),
                                               aux[v, ..., 0].view(np.float32).reshape(-1), want_abs=True)
        per_view[v]["proj_grads"] = check_pg_explained(gpg[v], opg, absum, flags_bwd, label=f"{label} view {v}")
        ab = GRAD_ABS_REL * np.asarray(absum, np.float64)
        unc[:, 10] += ab[:, 2] * sig * (1.0 - sig)
        unc[:, 11:14] += ab[:, 8:11] * 0.2820948
        unc[:, 14:59] += np.repeat(ab[:, 8:11], 15, axis=1) * 1.1
        pipe.r.project_backward(pipe.g, pipe.pg, cams[v], grads, view_offset=v * pipe.stride * 48)
        ogv = oracle.project_backward(os_, gpg[v], ocams[v])
        alt += ogv
        per_view[v]["param_grads"] = check_param_grads(grads.readback(n).flat(), ogv, label=f"{label} view {v}")
    report["views"] = per_view
    if trainer:
        cfg = TrainConfig(n_views=V, width=W, height=H, tile_w=tl.tile_w, tile_h=tl.tile_h, depth_max=tl.depth_max,
                          exact_backward=(mode == 1), use_graph=True)
        g = GpuSplatBuffer.upload(ctx, scene)
        mo = AdamMomentBuffers(ctx, g.capacity)
        acc = ctx.storage_buffer_zeroed("acc", 4 * g.capacity)
        tr = Trainer(ctx, cfg)
        tr.set_targets(ctx.storage_buffer("targets", np.ascontiguousarray(tgt, np.float32)))
        tloss = tr.step(g, mo, acc, cams, 1)
        assert np.array_equal(tr.images().reshape(V, H, W, 4), img), "trainer and stage path render differently"
        assert abs(tloss - loss) <= 1e-5 * loss, (tloss, loss)
        # the oracle's gradient of its own images (GPU records and bins, the oracle's blends)
        ograds = np.zeros((n, 59), np.float64)
        for v in range(V):
            rv = ranges[v * T:(v + 1) * T].reshape(-1)
            oimg, oncon, otf = oracle.composite(rec[v], pay, rv, otl)
            _, odl = oracle.mse(oimg, tgt[v], 1.0 / V)
            opg2 = oracle.composite_backward(rec[v], pay, rv, otl, oimg.reshape(-1, 4), odl, mode,
                                             oncon.reshape(-1), otf.reshape(-1))
            ograds += oracle.project_backward(os_, opg2, ocams[v])
        want = adam_first_step(scene.flat(), ograds.astype(np.float32), BENCH_LRS)
        report["post_adam"] = check_post_adam(g.readback().flat(), want, ograds, flags_bwd | flags_fwd, alt, unc,
                                              BENCH_LRS, label=label)
    report["seconds"] = round(time.time() - t0, 1)
    return report
