"""The reference's own known-answer tests, run against the CPU oracle (no GPU).

Each test names the reference test it restates; the vectors come from
tests/golden/reference_kats.json (transcribed from the reference sources).
These pin the oracle before it is trusted as the checker of the CUDA path.
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest

KATS = json.loads((Path(__file__).parent / "golden" / "reference_kats.json").read_text())


def rec_of(mx, my, depth, radius, conic=(1.0, 0.0, 1.0), color=(1.0, 1.0, 1.0), opacity=1.0):
    return [mx, my, depth, radius, *conic, 1.0, *color, opacity]


def one_splat(O, pos, rot, ls, op, dc, rest=None):
    return O.OSplats([pos], [rot], [ls], [op], [dc], [rest if rest is not None else np.zeros(45)])


def test_cpu_oracle_centers_on_axis(oracle):
    k = KATS["cpu_oracle_centers_on_axis"]
    sp, cm, ex = k["splat"], k["camera"], k["expect"]
    s = one_splat(oracle, sp["pos"], sp["rot"], sp["log_scale"], sp["opacity_logit"], sp["sh_dc"])
    cam = oracle.camera(cm["eye"], cm["target"], cm["up"], cm["fov_y"], cm["width"], cm["height"], 1)
    for sfx in ("f32", "f64"):
        r = oracle.project(s, cam, sfx)[0]
        assert r[7] == ex["visible"]
        assert abs(r[0] - ex["mean"][0]) < ex["mean_tol"] and abs(r[1] - ex["mean"][1]) < ex["mean_tol"]
        assert abs(r[2] - ex["depth"]) < ex["depth_tol"]
        assert ex["radius_open_interval"][0] < r[3] < ex["radius_open_interval"][1]
        assert abs(r[5]) < ex["conic_b_abs_max"]
        assert abs(r[4] - r[6]) < ex["conic_a_minus_c_abs_max"]


def test_composite_single_splat_renders_gaussian(oracle):
    k = KATS["composite_single_splat_renders_gaussian"]
    r, t, ex = k["record"], k["tiling"], k["expect"]
    rec = np.array([rec_of(*r["mean_xy"], r["depth"], r["radius"], r["conic"], r["color"], r["opacity"])], np.float32)
    tl = oracle.tiling(t["width"], t["height"], t["tile_size"], depth_max=t["depth_max"])
    _, pay, ranges = oracle.bin_ref(rec, tl)
    img, _, _ = oracle.composite(rec, pay, ranges, tl)
    c = img[ex["centre_xy"][1], ex["centre_xy"][0]]
    n = img[ex["near_xy"][1], ex["near_xy"][0]]
    e = img[ex["edge_xy"][1], ex["edge_xy"][0]]
    assert c[0] > ex["centre_rgb_min"] and c[3] > ex["centre_alpha_min"]
    assert n[0] > ex["near_rgb_min"] and n[0] < c[0] + 1e-3
    assert e[0] < ex["edge_rgb_max"] and e[3] < ex["edge_alpha_max"]
    for d in range(ex["diag_steps"]):
        assert img[32 + d, 32 + d, 3] <= c[3] + ex["diag_tol"]


def test_backward_accumulates_per_splat_gradients(oracle):
    k = KATS["backward_accumulates_per_splat_gradients"]
    r, t, ex = k["record"], k["tiling"], k["expect"]
    rec = np.array([rec_of(*r["mean_xy"], r["depth"], r["radius"], r["conic"], r["color"], r["opacity"])], np.float32)
    tl = oracle.tiling(t["width"], t["height"], t["tile_size"], depth_max=t["depth_max"])
    _, pay, ranges = oracle.bin_ref(rec, tl)
    img, ncon, tfin = oracle.composite(rec, pay, ranges, tl)
    dl = np.tile(np.array(k["dl_dc"], np.float32), (t["width"] * t["height"], 1))
    for mode in (0, 1):
        g = oracle.composite_backward(rec, pay, ranges, tl, img, dl, mode, ncon, tfin)[0]
        assert min(g[8], g[9], g[10]) > ex["dcolor_min"]
        assert g[2] > ex["dopacity_min"]
        assert g[4] < ex["dconic_a_max"] and g[6] < ex["dconic_c_max"]
        assert abs(g[0]) < ex["dmean_abs_max"] and abs(g[1]) < ex["dmean_abs_max"]


def test_four_splats_bin_to_expected_tiles(oracle):
    k = KATS["four_splats_bin_to_expected_tiles"]
    rec = np.array([rec_of(*r) for r in k["records"]], np.float32)
    t, ex = k["tiling"], k["expect"]
    tl = oracle.tiling(t["width"], t["height"], t["tile_size"], depth_max=t["depth_max"])
    keys, pay, ranges = oracle.bin_ref(rec, tl)
    assert len(keys) == ex["total_pairs"] and ranges.shape[0] == ex["num_tiles"]
    assert list(keys >> 16) == ex["tiles"]
    nz = [[i, int(b), int(e)] for i, (b, e) in enumerate(ranges) if e > b]
    assert nz == ex["ranges"]
    assert list(pay) == ex["payloads"]
    # the 64-bit native key layout gives the same order
    k64, p64, r64 = oracle.bin64(rec, 1, tl)
    assert list(p64) == ex["payloads"] and np.array_equal(r64, ranges)


def test_two_splats_same_tile_sorted_by_depth(oracle):
    k = KATS["two_splats_same_tile_sorted_by_depth"]
    rec = np.array([rec_of(*r) for r in k["records"]], np.float32)
    t, ex = k["tiling"], k["expect"]
    tl = oracle.tiling(t["width"], t["height"], t["tile_size"], depth_max=t["depth_max"])
    keys, pay, ranges = oracle.bin_ref(rec, tl)
    assert len(keys) == ex["total_pairs"]
    assert list(keys >> 16) == ex["tiles"]
    assert list(pay) == ex["payloads"]
    assert list(ranges[5]) == ex["tile5_range"]


def _fd_setup(oracle, sfx):
    k = KATS["finite_diff_matches_analytic"]
    sp, cm, t = k["splat"], k["camera"], k["tiling"]
    rest = np.zeros(45)
    for i, v in sp["sh_rest"].items():
        rest[int(i)] = v
    base = dict(pos=np.array(sp["pos"], float), rot=np.array(sp["rot"], float), ls=np.array(sp["log_scale"], float),
                op=sp["opacity_logit"], dc=np.array(sp["sh_dc"], float), rest=rest)
    cam = oracle.camera(cm["eye"], cm["target"], cm["up"], cm["fov_y"], cm["width"], cm["height"], 1)
    tl = oracle.tiling(cm["width"], cm["height"], t["tile_size"], depth_max=t["depth_max"])
    return k, base, cam, tl


def _fd_loss(oracle, p, cam, tl, sfx):
    s = one_splat(oracle, p["pos"], p["rot"], p["ls"], p["op"], p["dc"], p["rest"])
    rec = oracle.project(s, cam, sfx)
    _, pay, ranges = oracle.bin_ref(rec.astype(np.float32), tl)
    img, _, _ = oracle.composite(rec, pay, ranges, tl, sfx)
    return float(img[..., :3].astype(np.float64).sum())


def _fd_analytic(oracle, p, cam, tl, sfx, mode):
    s = one_splat(oracle, p["pos"], p["rot"], p["ls"], p["op"], p["dc"], p["rest"])
    rec = oracle.project(s, cam, sfx)
    _, pay, ranges = oracle.bin_ref(rec.astype(np.float32), tl)
    img, ncon, tfin = oracle.composite(rec, pay, ranges, tl, sfx)
    dl = np.tile(np.array([1.0, 1.0, 1.0, 0.0]), (tl.width * tl.height, 1))
    pg = oracle.composite_backward(rec, pay, ranges, tl, img, dl, mode, ncon, tfin, sfx)
    return oracle.project_backward(s, pg, cam, sfx)[0]


FD_PARAMS = {"sh_dc.r": ("dc", 0, 11), "opacity": ("op", None, 10), "sh_rest[0]": ("rest", 0, 14),
             "pos.x": ("pos", 0, 0), "log_scale.x": ("ls", 0, 7)}


@pytest.mark.parametrize("sfx", ["f32", "f64"])
@pytest.mark.parametrize("mode", [0, 1])
def test_finite_diff_matches_analytic(oracle, sfx, mode):
    """backward_finite_diff.rs:173-246 with the reference's tolerances, on both
    backward modes (the single splat never saturates, so ref == exact here)."""
    k, base, cam, tl = _fd_setup(oracle, sfx)
    g = _fd_analytic(oracle, base, cam, tl, sfx, mode)
    eps = k["eps"]
    for name, (field, idx, col) in FD_PARAMS.items():
        vals = []
        for sgn in (1, -1):
            p = {kk: (v.copy() if isinstance(v, np.ndarray) else v) for kk, v in base.items()}
            if idx is None:
                p[field] = p[field] + sgn * eps
            else:
                p[field][idx] += sgn * eps
            vals.append(_fd_loss(oracle, p, cam, tl, sfx))
        num = (vals[0] - vals[1]) / (2 * eps)
        rel, ab = k["checks"][name]
        a = float(g[col])
        assert abs(a - num) <= ab or abs(a - num) <= rel * (abs(a) + abs(num)), (name, a, num)


def test_adam_basics(oracle):
    """adam.rs:119-149: the step moves against the gradient, moments persist."""
    p, m, v = oracle.adam_step([1.0, 2.0, 3.0], [1.0, 1.0, 1.0], np.zeros(3), np.zeros(3), 1.6e-4, 1)
    assert np.all(p < np.array([1.0, 2.0, 3.0], np.float32))
    pp, mm, vv = np.zeros(1, np.float32), np.zeros(1, np.float32), np.zeros(1, np.float32)
    for t in range(1, 11):
        pp, mm, vv = oracle.adam_step(pp, [1.0], mm, vv, 1.6e-4, t)
    assert mm[0] > 0 and vv[0] > 0


def test_adam_oracle_matches_reference_formula(oracle):
    """adam.rs:70-90 evaluated in numpy float32, operation by operation."""
    rng = np.random.default_rng(3)
    n = 257
    p0 = rng.normal(size=n).astype(np.float32)
    g = rng.normal(size=n).astype(np.float32)
    m = rng.normal(size=n).astype(np.float32) * 0.1
    v = np.abs(rng.normal(size=n)).astype(np.float32) * 0.01
    t = 7
    b1, b2, lr, eps = np.float32(0.9), np.float32(0.999), np.float32(1.6e-4), np.float32(1e-15)
    bc1 = np.float32(1) - np.float32(oracle.lib().oracle_powi_f32(0.9, t))
    bc2 = np.float32(1) - np.float32(oracle.lib().oracle_powi_f32(0.999, t))
    mn = b1 * m + (np.float32(1) - b1) * g
    vn = b2 * v + (np.float32(1) - b2) * g * g
    pn = p0 - lr * (mn / bc1) / (np.sqrt(vn / bc2) + eps)
    po, mo, vo = oracle.adam_step(p0, g, m, v, 1.6e-4, t)
    assert np.array_equal(mo, mn) and np.array_equal(vo, vn) and np.array_equal(po, pn)


def _densify_kat_buffers(oracle, k):
    sp = k["splats"]
    s = oracle.OSplats([x["pos"] for x in sp], [x["rot"] for x in sp], [x["scale"] for x in sp],
                       [x["opacity"] for x in sp], [x["dc"] for x in sp], np.zeros((len(sp), 45)), capacity=16)
    m = oracle.OSplats.zeros(len(sp), 16)
    v = oracle.OSplats.zeros(len(sp), 16)
    return s, m, v


def test_densify_clones_small_and_splits_large(oracle):
    k = KATS["densify_clones_small_and_splits_large"]
    s, m, v = _densify_kat_buffers(oracle, k)
    acc = np.zeros(3 + 2 * k["max_splats"], np.float32)
    acc[:3] = k["grad_acc"]
    c = oracle.densify(s, m, v, acc, k["grad_count"], k["threshold"], k["split_thr"], k["max_splats"], k["iter"])
    ex = k["expect"]
    assert c == (ex["cloned"], ex["split_children"], ex["removed"])
    assert s.n == ex["len"] and m.n == ex["len"] and v.n == ex["len"]


def test_prune_drops_low_opacity_splats(oracle):
    k = KATS["prune_drops_low_opacity_splats"]
    n = len(k["opacities"])
    s = oracle.OSplats([[i, i, i] for i in range(n)], [[1, 0, 0, 0]] * n, [[-1, -1, -1]] * n, k["opacities"],
                       np.zeros((n, 3)), np.zeros((n, 45)), capacity=n)
    m, v = oracle.OSplats.zeros(n), oracle.OSplats.zeros(n)
    acc = np.array(k["grad_acc"], np.float32)
    removed = oracle.prune(s, m, v, acc, k["threshold"])
    ex = k["expect"]
    assert removed == ex["removed"] and s.n == ex["len"]
    assert np.allclose(s.get()[3], ex["survivor_opacity"])


def swap_remove_sources(rm: np.ndarray) -> list[int]:
    """Closed form of descending swap_remove used by the CUDA compaction: with
    excl the exclusive prefix count of removals and m their number, the
    removal of descending rank k receives the element at position n-k; a
    removed position q there resolves to n - m + excl[q] (strictly larger),
    until a survivor is reached."""
    n = len(rm)
    excl = np.concatenate([[0], np.cumsum(rm)[:-1]]).astype(int) if n else np.zeros(0, int)
    m = int(rm.sum())
    src = list(range(n - m))
    for j in range(n - m):
        if rm[j]:
            q = n - (m - excl[j])
            while rm[q]:
                q = n - m + excl[q]
            src[j] = q
    return src


def test_swap_remove_order_closed_form(oracle):
    """The rule the CUDA prune relies on, checked against the oracle's literal
    swap_remove sequence (train.rs:572-602) on random removal sets."""
    rng = np.random.default_rng(11)
    for trial in range(400):
        n = int(rng.integers(1, 80))
        ops = np.where(rng.random(n) < rng.random(), -10.0, 2.0).astype(np.float32)
        s = oracle.OSplats(np.arange(n)[:, None].repeat(3, 1), [[1, 0, 0, 0]] * n, np.zeros((n, 3)), ops,
                           np.zeros((n, 3)), np.zeros((n, 45)))
        oracle.prune(s, None, None, None, -5.3)
        got = s.get()[0][:, 0].astype(int)
        assert list(got) == swap_remove_sources(ops < -5.3), (trial, ops)


def test_oracle_ply_roundtrip(oracle, tmp_path):
    k = KATS["ply_write_then_read_roundtrip"]["gaussian"]
    s = oracle.OSplats([k["pos"]], [k["rotation"]], [k["scale"]], [k["opacity"]], [k["sh_dc"]],
                       [np.arange(45) * 0.1])
    path = tmp_path / "a.ply"
    assert oracle.write_ply(path, s) == 0
    r, back = oracle.read_ply(path, 4)
    assert r == 1
    assert np.array_equal(back.flat(), s.flat())


def test_mse_matches_reference_formula(oracle):
    """loss.rs:163-179: dL/dC = 2 (p - t) / (3 W H), loss = sum (p-t)^2 / (3 W H)."""
    rng = np.random.default_rng(5)
    P = 97
    pred = rng.random((P, 4)).astype(np.float32)
    tgt = rng.random((P, 3)).astype(np.float32)
    loss, dl = oracle.mse(pred, tgt)
    d = pred[:, :3] - tgt
    inv_n = np.float32(2.0) / np.float32(P * 3)
    assert np.array_equal(dl.reshape(P, 4)[:, :3], d * inv_n)
    per_pixel = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2]).astype(np.float64)  # f32, then f64 sum
    assert abs(loss - float(per_pixel.sum() / (P * 3))) < 1e-12


# ---- SSIM and the combined loss: the reference's loss tests (loss.rs:412-600,
# tests/loss_tests.rs:10-125) run on the oracle's restatement
def _rgba(rgb):
    rgb = np.asarray(rgb, np.float32).reshape(-1, 3)
    return np.concatenate([rgb, np.zeros((len(rgb), 1), np.float32)], axis=1)


def _checkerboard(w, h, scale):
    out = []
    for y in range(h):
        for x in range(w):
            v = scale if (x + y) % 2 == 0 else 0.0
            out.append((v, v * 0.5, v * 0.25))
    return np.array(out, np.float32)


def _ramp(w, h, scale):
    n = w * h
    f = np.arange(n, dtype=np.float32) / np.float32(n)
    return np.stack([scale * f, scale * (1 - f), scale * (0.3 + 0.4 * f)], axis=1).astype(np.float32)


def _lcg_noise(img, seed):
    out = img.copy()
    s = seed
    for i in range(len(out)):
        s = (s * 1103515245 + 12345) & 0xFFFFFFFF
        out[i] += np.float32(((s >> 16) / 65535.0 - 0.5) * 0.4)
    return out


@pytest.mark.parametrize("img", [_checkerboard(8, 8, 0.7), _ramp(8, 8, 0.7)])
def test_ssim_is_zero_loss_for_identical_images(oracle, img):
    loss, dl = oracle.ssim(_rgba(img), img, 8, 8)
    assert abs(loss) < 1e-5
    assert np.all(np.linalg.norm(dl.reshape(-1, 4)[:, :3], axis=1) < 1e-4)


@pytest.mark.parametrize("img,seed", [(_checkerboard(8, 8, 0.7), 1), (_ramp(8, 8, 0.7), 12345)])
def test_ssim_loss_grows_with_noise(oracle, img, seed):
    clean, _ = oracle.ssim(_rgba(img), img, 8, 8)
    dirty, _ = oracle.ssim(_rgba(_lcg_noise(img, seed)), img, 8, 8)
    assert dirty > clean


def test_ssim_gradient_matches_finite_diff(oracle):
    n = 64
    f = np.arange(n, dtype=np.float32) / np.float32(n)
    pred = np.stack([0.3 + 0.4 * f, 0.5 - 0.3 * f, 0.2 + 0.6 * f], 1).astype(np.float32)
    tgt = np.stack([0.4 + 0.3 * f, 0.6 - 0.4 * f, 0.3 + 0.5 * f], 1).astype(np.float32)
    _, an = oracle.ssim(_rgba(pred), tgt, 8, 8)
    an = an.reshape(-1, 4)
    eps = np.float32(1e-3)
    for i in range(n):
        for ch in range(3):
            pp, pm = pred.copy(), pred.copy()
            pp[i, ch] += eps
            pm[i, ch] -= eps
            lp, _ = oracle.ssim(_rgba(pp), tgt, 8, 8)
            lm, _ = oracle.ssim(_rgba(pm), tgt, 8, 8)
            fd = (np.float32(lp) - np.float32(lm)) / (2 * eps)
            assert abs(fd - an[i, ch]) < 5e-3


def _pair(kind):
    n = 64
    f = np.arange(n, dtype=np.float32) / np.float32(n)
    if kind == "a":
        p = np.stack([f, 1 - f, np.full(n, 0.3, np.float32)], 1)
        t = np.stack([f * 0.9, 1 - f * 1.1, np.full(n, 0.4, np.float32)], 1)
    else:
        p = np.stack([0.2 + f, np.full(n, 0.4, np.float32), 0.5 - f * 0.3], 1)
        t = np.stack([0.25 + f * 0.9, np.full(n, 0.5, np.float32), 0.55 - f * 0.2], 1)
    return p.astype(np.float32), t.astype(np.float32)


def test_combined_lambda_zero_is_pure_mse_and_one_is_pure_ssim(oracle):
    p, t = _pair("a")
    mse, gm = oracle.mse(_rgba(p), t)
    total, mc, sc, g = oracle.combined(_rgba(p), t, 8, 8, 0.0)
    assert total == mse and mc == mse and sc == 0.0
    assert np.max(np.abs(g - gm)) < 1e-9
    ssim, gs = oracle.ssim(_rgba(p), t, 8, 8)
    total, mc, sc, g = oracle.combined(_rgba(p), t, 8, 8, 1.0)
    assert total == ssim and mc == 0.0 and sc == ssim
    assert np.max(np.abs(g - gs)) < 1e-9


def test_combined_gradient_is_lambda_weighted_sum(oracle):
    p, t = _pair("b")
    lam = np.float32(0.2)
    _, gm = oracle.mse(_rgba(p), t)
    _, gs = oracle.ssim(_rgba(p), t, 8, 8)
    _, _, _, g = oracle.combined(_rgba(p), t, 8, 8, float(lam))
    want = gm * (np.float32(1) - lam) + gs * lam
    assert np.max(np.linalg.norm((g - want).reshape(-1, 4), axis=1)) < 1e-6


def test_fp64_adjoint_matches_central_differences_on_64_random_parameters(oracle):
    """The adjoint check on the oracle's FP64 instantiation:
    central differences (h = 1e-3, FP64 loss) on 64 random parameters of a
    1000-splat 64x64 scene, rotations included (tests/fd64.py states the
    bounds and the counted exceptions)."""
    from tests.fd64 import Scene64, compare
    s = Scene64(oracle)
    adj, rec = s.adjoint_f64()
    _, summary = compare(s, adj, s.draw(adj), rec)
    print(summary)
