"""GPU parity of the rasteriser path against the CPU oracle, through the C ABI.

Stages are compared on shared inputs: the oracle bins the GPU's projected
records, blends the GPU's bins, and differentiates the GPU's images, so
integer results (bins, sort order, ranges) must match bit for bit and float
results within the tolerances of tests/util.py:
  images  <= 1e-4 absolute on every pixel except those whose walk passes
          within a stated relative margin of a blend threshold (alpha vs
          1/255 or 0.99, T vs 1e-4, the reference backward's T vs 1.0001),
          counted and at most 0.1 % of the pixels
  grads   <= 1e-3 relative per component plus 1e-4 of the sum of the terms'
          magnitudes, except splats in the walk of such a pixel
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from nanotracer_b200 import CameraUniform, GpuSplatBuffer, PrefixScan, RadixSort, Rasterizer, TileBinner, TilingParams
from nanotracer_b200._lib import SC_BWD_EXACT, SC_BWD_REF, SC_KEYS_NATIVE64, SC_KEYS_REF32
from nanotracer_b200.scene import FOV_Y, orbit_pose, orbit_views, random_scene

from tests.util import GpuPipe, check_image_explained, check_param_grads, check_pg_explained, margins, small_scene

pytestmark = pytest.mark.gpu
KATS = json.loads((Path(__file__).parent / "golden" / "reference_kats.json").read_text())


def _osplats(oracle, scene):
    return oracle.OSplats.from_buffer(scene)


def _ocam(oracle, cam: CameraUniform):
    return oracle.camera_from_struct(bytes(cam.c))


def _otl(oracle, tl: TilingParams):
    return oracle.tiling(tl.width, tl.height, tl.tile_w, tl.tile_h, tl.depth_max)


# ------------------------------------------------------------------ projection
def test_wgsl_matches_cpu_oracle_unit_splat(ctx, oracle):
    """raster.rs:1217-1265 with its tolerances."""
    k = KATS["cpu_oracle_centers_on_axis"]
    tol = KATS["wgsl_matches_cpu_oracle_tolerances"]["tol"]
    sp, cm = k["splat"], k["camera"]
    from nanotracer_b200 import SplatBuffer
    s = SplatBuffer([sp["pos"]], [sp["rot"]], [sp["log_scale"]], [sp["opacity_logit"]], [sp["sh_dc"]],
                    np.zeros((1, 45)))
    cam = CameraUniform.from_pose(cm["eye"], cm["target"], cm["up"], cm["fov_y"], cm["width"], cm["height"], 1)
    pipe = GpuPipe(ctx, s, cam, TilingParams(256, 256, 16, 100.0))
    g = pipe.project()[0, 0]
    o = oracle.project(_osplats(oracle, s), _ocam(oracle, cam))[0]
    assert g[7] == 1.0
    assert abs(g[0] - o[0]) < tol["mean"] and abs(g[1] - o[1]) < tol["mean"]
    assert abs(g[2] - o[2]) < tol["depth"] and abs(g[3] - o[3]) < tol["radius"]
    assert np.all(np.abs(g[4:7] - o[4:7]) < tol["conic"])
    assert np.all(np.abs(g[8:11] - o[8:11]) < tol["color"])
    assert abs(g[11] - o[11]) < tol["opacity"]


@pytest.mark.parametrize("n_views", [1, 3])
def test_projection_parity_small_scene(ctx, oracle, n_views):
    scene, _, tl = small_scene()
    cams = [CameraUniform.from_pose(*p, FOV_Y, tl.width, tl.height, len(scene)) for p in orbit_views(n_views, 5)]
    pipe = GpuPipe(ctx, scene, cams, tl)
    gpu = pipe.project()
    os_ = _osplats(oracle, scene)
    for v, cam in enumerate(cams):
        o = oracle.project(os_, _ocam(oracle, cam))
        g = gpu[v]
        same_vis = g[:, 7] == o[:, 7]
        assert same_vis.mean() >= 0.999
        m = same_vis & (o[:, 7] == 1)
        assert np.abs(g[m, 0:2] - o[m, 0:2]).max() < 1e-3
        assert np.allclose(g[m, 2], o[m, 2], rtol=1e-5)
        assert np.abs(g[m, 3] - o[m, 3]).max() <= 1.0
        assert (g[m, 3] == o[m, 3]).mean() > 0.999
        assert np.allclose(g[m, 4:7], o[m, 4:7], rtol=1e-4, atol=1e-7)
        assert np.abs(g[m, 8:11] - o[m, 8:11]).max() < 1e-5
        assert np.abs(g[m, 11] - o[m, 11]).max() < 1e-6
        # culled records are all zeros like the reference's default record
        assert np.all(g[g[:, 7] == 0] == 0)


def test_projection_against_fp64_oracle(ctx, oracle):
    """The f32 GPU projection of ordinary (small-scene) splats against the FP64
    oracle: the error statement of the default f32 arithmetic."""
    scene, cam, tl = small_scene(2000)
    pipe = GpuPipe(ctx, scene, cam, tl)
    g = pipe.project()[0]
    o = oracle.project(_osplats(oracle, scene), _ocam(oracle, cam), "f64")
    m = (g[:, 7] == 1) & (o[:, 7] == 1)
    rel = np.abs(g[m, 4:7] - o[m, 4:7]) / np.maximum(np.abs(o[m, 4:7]), 1e-6)
    assert np.median(rel) < 1e-5


def test_roundtrip_upload_readback_bit_exact(ctx):
    """splat_gpu.rs:451-473."""
    scene = random_scene(1234, seed=3)
    g = GpuSplatBuffer.upload(ctx, scene)
    back = g.readback()
    assert np.array_equal(back.flat(), scene.flat())
    scene2 = random_scene(1234, seed=4)
    g.sync_from(scene2)
    assert np.array_equal(g.readback().flat(), scene2.flat())


def test_bf16_rest_storage_rounds_to_nearest_even(ctx):
    import torch
    scene = random_scene(300, seed=5)
    g = GpuSplatBuffer.upload(ctx, scene, bf16_rest=True)
    back = g.readback()
    want = torch.from_numpy(scene.sh_rest).to(torch.bfloat16).float().numpy()
    assert np.array_equal(back.sh_rest, want)
    assert np.array_equal(back.flat()[:, :14], scene.flat()[:, :14])


# ------------------------------------------------------------------ binning / sort / scan
def _upload_records(ctx, recs):
    arr = np.zeros((len(recs), 12), np.float32)
    for i, r in enumerate(recs):
        arr[i, :4] = r
        arr[i, 4:] = [1.0, 0.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0]
    return ctx.storage_buffer("projected", arr), arr


@pytest.mark.parametrize("key_mode", [SC_KEYS_REF32, SC_KEYS_NATIVE64])
def test_four_splats_bin_to_expected_tiles(ctx, key_mode):
    k = KATS["four_splats_bin_to_expected_tiles"]
    buf, _ = _upload_records(ctx, k["records"])
    t, ex = k["tiling"], k["expect"]
    res = TileBinner(ctx).bin(buf, 4, TilingParams(t["width"], t["height"], t["tile_size"], t["depth_max"]),
                              key_mode=key_mode)
    assert res.total_pairs == ex["total_pairs"] and res.num_tiles == ex["num_tiles"]
    keys = res.sorted_keys()
    tiles = list(keys >> (16 if key_mode == SC_KEYS_REF32 else 32))
    assert tiles == ex["tiles"]
    ranges = res.tile_ranges()
    nz = [[i, int(b), int(e)] for i, (b, e) in enumerate(ranges) if e > b]
    assert nz == ex["ranges"]
    assert list(res.sorted_payloads()) == ex["payloads"]


def test_two_splats_same_tile_sorted_by_depth(ctx):
    k = KATS["two_splats_same_tile_sorted_by_depth"]
    buf, _ = _upload_records(ctx, k["records"])
    t, ex = k["tiling"], k["expect"]
    res = TileBinner(ctx).bin(buf, 2, TilingParams(t["width"], t["height"], t["tile_size"], t["depth_max"]))
    assert res.total_pairs == 2
    assert list(res.sorted_keys() >> 16) == ex["tiles"]
    assert list(res.sorted_payloads()) == ex["payloads"]
    assert list(res.tile_ranges()[5]) == ex["tile5_range"]


def test_empty_scene_bins_and_composite(ctx):
    """tile_binner.rs:247-259 empty fast path: no pairs, every range (0,0), black image."""
    buf = ctx.storage_buffer("projected", np.zeros((3, 12), np.float32))
    tl = TilingParams(64, 48, 16, 100.0)
    res = TileBinner(ctx).bin(buf, 3, tl)
    assert res.total_pairs == 0 and np.all(res.tile_ranges() == 0)
    r = Rasterizer(ctx)
    img = r.alloc_image(64, 48)
    r.composite(buf, res, img, tl, stride=3)
    assert np.all(img.readback(np.float32) == 0)


@pytest.mark.parametrize("key_mode", [SC_KEYS_REF32, SC_KEYS_NATIVE64])
@pytest.mark.parametrize("tile", [(16, 16), (8, 8), (32, 8)])
def test_bins_bit_exact_vs_oracle(ctx, oracle, key_mode, tile):
    scene, cam, tl0 = small_scene()
    tl = TilingParams(tl0.width, tl0.height, tile[0], tl0.depth_max, tile_h_override=tile[1])
    pipe = GpuPipe(ctx, scene, cam, tl, key_mode=key_mode)
    rec = pipe.project()[0]
    keys, pay, ranges = pipe.bin()
    otl = _otl(oracle, tl)
    if key_mode == SC_KEYS_REF32:
        ok, op, orr = oracle.bin_ref(rec, otl)
    else:
        ok, op, orr = oracle.bin64(rec, 1, otl)
    assert len(keys) == len(ok)
    assert np.array_equal(keys, ok)
    assert np.array_equal(pay, op)
    assert np.array_equal(ranges, orr)


def test_bins_multiview_native64_vs_oracle(ctx, oracle):
    scene, _, tl = small_scene(3000)
    cams = [CameraUniform.from_pose(*p, FOV_Y, tl.width, tl.height, len(scene)) for p in orbit_views(4, 2)]
    pipe = GpuPipe(ctx, scene, cams, tl, key_mode=SC_KEYS_NATIVE64)
    rec = pipe.project()  # (V, n, 12)
    keys, pay, ranges = pipe.bin()
    ok, op, orr = oracle.bin64(rec.reshape(-1, 12), 4, _otl(oracle, tl))
    assert np.array_equal(keys, ok) and np.array_equal(pay, op) and np.array_equal(ranges, orr)


def _lcg(seed, n, mod=None):
    out = np.empty(n, np.uint32)
    s = seed
    for i in range(n):
        s = (s * 1664525 + 1013904223) & 0xFFFFFFFF
        out[i] = s % mod if mod else s
    return out


def _sort_gpu(ctx, keys, vals, key_bits, key_bytes):
    ka = ctx.storage_buffer("ka", keys)
    va = ctx.storage_buffer("va", vals)
    kb = ctx.storage_buffer_zeroed("kb", keys.nbytes)
    vb = ctx.storage_buffer_zeroed("vb", vals.nbytes)
    RadixSort(ctx).sort(ka, va, kb, vb, len(keys), key_bits, key_bytes)
    return ka.readback(keys.dtype), va.readback(np.uint32)


def test_sort_small_array_stable(ctx):
    k = KATS["sort_small_array_stable"]
    sk, sv = _sort_gpu(ctx, np.array(k["keys"], np.uint32), np.array(k["vals"], np.uint32), 32, 4)
    assert list(sk) == k["expect"]["keys"] and list(sv[:2]) == k["expect"]["vals_prefix"]


def test_sort_random_u32_with_payload(ctx):
    k = KATS["sort_random_u32_with_payload"]
    keys = _lcg(k["lcg"]["seed"], k["n"])
    vals = np.arange(k["n"], dtype=np.uint32)
    sk, sv = _sort_gpu(ctx, keys, vals, 32, 4)
    assert np.array_equal(sk, keys[sv]) and np.all(sk[1:] >= sk[:-1])
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(sv, order)


# 9 bits: one 9-bit pass; the others 8-bit passes, with a narrower last digit
# for 7, 13, 17, 26, 35 and 44 bits
@pytest.mark.parametrize("n,bits,key_bytes", [(1, 8, 4), (4097, 13, 4), (3_000_001, 16, 4), (2_500_003, 35, 8),
                                              (1_000_000, 64, 8), (777_777, 7, 8), (2_000_003, 9, 4),
                                              (1_000_001, 17, 4), (999_999, 26, 4), (500_001, 44, 8)])
def test_sort_stable_vs_numpy(ctx, n, bits, key_bytes):
    rng = np.random.default_rng(n + bits)
    dt = np.uint32 if key_bytes == 4 else np.uint64
    keys = rng.integers(0, 1 << bits, n, dtype=np.uint64, endpoint=False) if bits < 64 else \
        rng.integers(0, np.iinfo(np.uint64).max, n, dtype=np.uint64, endpoint=True)
    keys = keys.astype(dt)
    vals = np.arange(n, dtype=np.uint32)
    sk, sv = _sort_gpu(ctx, keys, vals, bits, key_bytes)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(sv, order.astype(np.uint32))
    assert np.array_equal(sk, keys[order])


def test_scan_all_ones_yields_indices(ctx):
    buf = ctx.storage_buffer("s", np.ones(1000, np.uint32))
    tot = ctx.storage_buffer_zeroed("t", 8)
    PrefixScan(ctx).scan(buf, 1000, tot)
    assert np.array_equal(buf.readback(np.uint32), np.arange(1000, dtype=np.uint32))
    assert tot.readback(np.uint64)[0] == 1000


@pytest.mark.parametrize("n", [70_000, 1, 4096, 4097, 10_000_019])
def test_scan_random_matches_cpu_reference(ctx, n):
    x = _lcg(0x12345678, n, 17) if n == 70_000 else np.random.default_rng(n).integers(0, 300, n).astype(np.uint32)
    buf = ctx.storage_buffer("s", x)
    tot = ctx.storage_buffer_zeroed("t", 8)
    PrefixScan(ctx).scan(buf, n, tot)
    ex = np.concatenate([[0], np.cumsum(x.astype(np.uint64))[:-1]]).astype(np.uint32)
    assert np.array_equal(buf.readback(np.uint32), ex)
    assert tot.readback(np.uint64)[0] == int(x.astype(np.uint64).sum())


# ------------------------------------------------------------------ blending
def test_composite_single_splat_renders_gaussian(ctx):
    k = KATS["composite_single_splat_renders_gaussian"]
    r, t, ex = k["record"], k["tiling"], k["expect"]
    rec = np.array([[*r["mean_xy"], r["depth"], r["radius"], *r["conic"], r["visible"], *r["color"], r["opacity"]]],
                   np.float32)
    buf = ctx.storage_buffer("p", rec)
    tl = TilingParams(t["width"], t["height"], t["tile_size"], t["depth_max"])
    res = TileBinner(ctx).bin(buf, 1, tl)
    rz = Rasterizer(ctx)
    img = rz.alloc_image(64, 64)
    rz.composite(buf, res, img, tl, stride=1)
    px = img.readback(np.float32).reshape(64, 64, 4)
    c, n, e = px[32, 32], px[34, 34], px[0, 0]
    assert c[0] > ex["centre_rgb_min"] and c[3] > ex["centre_alpha_min"]
    assert ex["near_rgb_min"] < n[0] < c[0] + 1e-3
    assert e[0] < ex["edge_rgb_max"] and e[3] < ex["edge_alpha_max"]
    for d in range(16):
        assert px[32 + d, 32 + d, 3] <= c[3] + 1e-3


@pytest.mark.parametrize("mode", [SC_BWD_REF, SC_BWD_EXACT])
def test_backward_accumulates_per_splat_gradients(ctx, mode):
    k = KATS["backward_accumulates_per_splat_gradients"]
    r, t, ex = k["record"], k["tiling"], k["expect"]
    rec = np.array([[*r["mean_xy"], r["depth"], r["radius"], *r["conic"], r["visible"], *r["color"], r["opacity"]]],
                   np.float32)
    buf = ctx.storage_buffer("p", rec)
    tl = TilingParams(t["width"], t["height"], t["tile_size"], t["depth_max"])
    res = TileBinner(ctx).bin(buf, 1, tl)
    rz = Rasterizer(ctx)
    img, aux = rz.alloc_image(32, 32), rz.alloc_aux(32, 32)
    rz.composite(buf, res, img, tl, stride=1, aux=aux)
    dl = ctx.storage_buffer("dl", np.tile(np.array(k["dl_dc"], np.float32), (32 * 32, 1)))
    pg = ctx.storage_buffer_zeroed("pg", 48)
    rz.composite_backward(buf, res, img, dl, pg, tl, stride=1, mode=mode, aux=aux)
    g = pg.readback(np.float32)
    assert min(g[8], g[9], g[10]) > ex["dcolor_min"] and g[2] > ex["dopacity_min"]
    assert g[4] < ex["dconic_a_max"] and g[6] < ex["dconic_c_max"]
    assert abs(g[0]) < ex["dmean_abs_max"] and abs(g[1]) < ex["dmean_abs_max"]


@pytest.mark.parametrize("tile", [(16, 16), (8, 8), (32, 8)])
def test_composite_parity_small_scene(ctx, oracle, tile):
    scene, cam, tl0 = small_scene()
    tl = TilingParams(tl0.width, tl0.height, tile[0], tl0.depth_max, tile_h_override=tile[1])
    pipe = GpuPipe(ctx, scene, cam, tl)
    rec = pipe.project()[0]
    _, pay, ranges = pipe.bin()
    img, aux = pipe.composite()
    oimg, oncon, otf = oracle.composite(rec, pay, ranges.reshape(-1), _otl(oracle, tl))
    margin, _, _ = margins(oracle, rec, pay, ranges, _otl(oracle, tl), 1)
    print(check_image_explained(img[0], oimg, margin))
    near = margin < 1.0
    # last contributor and final T: equal except where a pixel's walk is near a threshold
    assert np.all((aux[0, ..., 1] == oncon) | near)
    tf = aux[0, ..., 0].view(np.float32)
    assert np.all((np.abs(tf - otf) <= 1e-5 * np.maximum(np.abs(otf), 1e-4)) | near)


def test_mse_loss_grad_vs_oracle(ctx, oracle):
    rng = np.random.default_rng(8)
    W, H, V = 96, 64, 2
    pred = rng.random((V, H, W, 4)).astype(np.float32)
    tgt = rng.random((V, H, W, 3)).astype(np.float32)
    rz = Rasterizer(ctx)
    pb, tb = ctx.storage_buffer("p", pred), ctx.storage_buffer("t", tgt)
    dl = ctx.storage_buffer_zeroed("dl", pred.nbytes)
    losses = rz.mse_loss_grad(pb, tb, TilingParams(W, H, 16), dl, n_views=V, scale=0.5)
    g = dl.readback(np.float32).reshape(V, H * W, 4)
    for v in range(V):
        l, od = oracle.mse(pred[v], tgt[v], 0.5)
        assert abs(losses[v] - l) <= 1e-12 + 1e-9 * l
        assert np.array_equal(g[v], od.reshape(-1, 4))


@pytest.mark.parametrize("mode", [SC_BWD_REF, SC_BWD_EXACT])
def test_composite_backward_parity_small_scene(ctx, oracle, mode):
    scene, cam, tl = small_scene()
    pipe = GpuPipe(ctx, scene, cam, tl)
    rec = pipe.project()[0]
    _, pay, ranges = pipe.bin()
    img, aux = pipe.composite()
    rng = np.random.default_rng(1)
    dl = (rng.normal(size=(tl.height * tl.width, 4)) * 1e-3).astype(np.float32)
    dl[:, 3] = 0
    gpu = pipe.backward(dl, mode)[0]
    ora, absum = oracle.composite_backward(rec, pay, ranges.reshape(-1), _otl(oracle, tl), img[0].reshape(-1, 4), dl,
                                           mode, aux[0, ..., 1].reshape(-1),
                                           aux[0, ..., 0].view(np.float32).reshape(-1), want_abs=True)
    _, flags, _ = margins(oracle, rec, pay, ranges, _otl(oracle, tl), mode)
    print(check_pg_explained(gpu, ora, absum, flags, label=f"small scene mode {mode}"))
    assert np.all(gpu[:, [3, 7, 11]] == 0)


def test_project_backward_parity_small_scene(ctx, oracle):
    from nanotracer_b200 import GradSplatBuffers
    scene, cam, tl = small_scene()
    pipe = GpuPipe(ctx, scene, cam, tl)
    pipe.project()
    pipe.bin()
    pipe.composite()
    rng = np.random.default_rng(2)
    dl = (rng.normal(size=(tl.height * tl.width, 4)) * 1e-3).astype(np.float32)
    pg = pipe.backward(dl, SC_BWD_EXACT)[0]
    grads = GradSplatBuffers(ctx, len(scene))
    pipe.r.project_backward(pipe.g, pipe.pg, cam, grads)
    gpu = grads.readback(len(scene)).flat()
    ora = oracle.project_backward(_osplats(oracle, scene), pg, _ocam(oracle, cam))
    print(check_param_grads(gpu, ora, rtol=1e-4))
    # accumulate=1 adds a second view's gradient
    pipe.r.project_backward(pipe.g, pipe.pg, cam, grads, accumulate=True)
    assert np.allclose(grads.readback(len(scene)).flat(), 2 * gpu, rtol=1e-6, atol=1e-12)


def test_tonemap_headless_buffer(ctx):
    img = np.array([[[0.0, 0.5, 1.0, 1.0], [4.0, -1.0, 0.002, 0.25]]], np.float32)
    b = ctx.storage_buffer("i", img)
    out = ctx.storage_buffer_zeroed("o", 2 * 4)
    Rasterizer(ctx).tonemap(b, 2, 1, out)
    px = out.readback(np.uint8).reshape(2, 4)

    def srgb(c):
        c = np.clip(c, 0, 1)
        return np.where(c > 0.0031308, 1.055 * c ** (1 / 2.4) - 0.055, c * 12.92)
    rgb = img[0, :, :3] / (1 + np.maximum(img[0, :, :3], 0))
    want = np.concatenate([np.round(np.clip(srgb(rgb), 0, 1) * 255), np.round(img[0, :, 3:] * 255)], 1)
    assert np.abs(px.astype(int) - want.astype(int)).max() <= 1


@pytest.mark.parametrize("bits,extent", [(13, 8160), (9, 510)])
def test_sort_on_low_key_bits_keeps_high_bits_in_input_order(ctx, bits, extent):
    """key_bits below the key width: ordered by the low bits only, stable, the
    high bits carried along (the trainer's (view << tile_bits) | tile pair keys,
    and its items: member mask and view above the 9 super-tile bits)."""
    rng = np.random.default_rng(11 + bits)
    n = 300_001
    keys = ((rng.integers(0, 1 << (32 - bits), n, dtype=np.uint64) << bits) |
            rng.integers(0, extent, n, dtype=np.uint64)).astype(np.uint32)
    vals = np.arange(n, dtype=np.uint32)
    sk, sv = _sort_gpu(ctx, keys, vals, bits, 4)
    order = np.argsort(keys & ((1 << bits) - 1), kind="stable")
    assert np.array_equal(sv, order.astype(np.uint32)) and np.array_equal(sk, keys[order])
