"""GPU parity of the optimiser step and of densify / prune against the oracle.

Adam parity follows tests/adam_gpu_parity.rs (params |d| < 1e-4, moments
|d| < 1e-5); the fp32 form here is held to 1e-6 relative.  Prune and densify
must reproduce the reference's swap_remove order exactly (integer layout is
bit-exact; moved parameters are bit-exact; split-children positions, which go
through log / cos / exp, within 1e-5).
"""
import json
import math
from pathlib import Path

import numpy as np
import pytest

from nanotracer_b200 import (AdamConfig, AdamGpu, AdamMomentBuffers, GpuSplatBuffer, GradSplatBuffers, SplatBuffer,
                             densify, prune_low_opacity)
from nanotracer_b200.scene import random_scene

pytestmark = pytest.mark.gpu
KATS = json.loads((Path(__file__).parent / "golden" / "reference_kats.json").read_text())


def _grad_fn(expr):
    return lambda t, i: eval(expr, {"sin": math.sin, "i": i, "t": t})


@pytest.mark.parametrize("run", range(5))
def test_adam_gpu_parity(ctx, oracle, run):
    k = KATS["adam_gpu_parity"]
    r = k["runs"][run]
    n, steps, f = r["n"], r["steps"], _grad_fn(r["grad"])
    cfg = AdamConfig()
    p = np.full(n, k["init_param"], np.float32)
    m = np.zeros(n, np.float32)
    v = np.zeros(n, np.float32)
    pb, mb, vb = ctx.storage_buffer("p", p), ctx.storage_buffer("m", m), ctx.storage_buffer("v", v)
    gb = ctx.storage_buffer_zeroed("g", 4 * n)
    adam = AdamGpu(ctx)
    for t in range(1, steps + 1):
        g = np.array([f(t, i) for i in range(n)], np.float32)
        p, m, v = oracle.adam_step(p, g, m, v, cfg.lr, t)
        gb.upload(g)
        adam.step(pb, gb, mb, vb, n, cfg.lr, t, cfg)
    gp, gm, gv = pb.readback(np.float32), mb.readback(np.float32), vb.readback(np.float32)
    assert np.abs(gp - p).max() < k["param_tol"] and np.abs(gm - m).max() < k["moment_tol"]
    assert np.abs(gv - v).max() < k["moment_tol"]
    assert np.allclose(gp, p, rtol=1e-6, atol=1e-7)


def test_step_all_matches_per_attribute_cpu(ctx, oracle):
    """adam_gpu_parity.rs:161-376: two lr groups over the whole parameter layout."""
    k = KATS["adam_gpu_parity"]
    n = 4
    rows = []
    for i in range(n):
        f = float(i)
        rest = 0.1 * f + 0.01 * np.arange(45)
        rows.append(np.concatenate([[f, f * 0.5 - 1.0, f * 2.0 + 0.25],
                                    [0.7 + 0.1 * f, 0.2 * f, -0.1 * f, 0.3 - 0.05 * f],
                                    [-1.0 - 0.1 * f, -1.2 + 0.05 * f, -0.9 * math.log(f + 1.0)],
                                    [-0.5 + 0.3 * f], [0.1 * f, 0.2 - 0.05 * f, 0.05 * f + 0.3], rest]))
    s = SplatBuffer.from_flat(np.array(rows, np.float32))
    grows = []
    for i in range(n):
        f = float(i)
        grows.append(np.concatenate([[0.10 + 0.001 * f, -0.07 - 0.002 * f, 0.03 + 0.0015 * f],
                                     [-0.05 + 0.001 * f, 0.04 - 0.002 * f, 0.06 + 0.0005 * f, -0.02 + 0.003 * f],
                                     [0.08 - 0.001 * f, -0.09 + 0.002 * f, 0.11 + 0.0005 * f], [-0.12 + 0.004 * f],
                                     [0.02 + 0.0007 * f, -0.03 - 0.0009 * f, 0.04 + 0.0011 * f],
                                     0.001 * (np.arange(45) + 1.0) + 0.0001 * f]))
    gflat = np.array(grows, np.float32)
    g = GpuSplatBuffer.upload(ctx, s)
    grads = GradSplatBuffers(ctx, n)
    grads.upload(SplatBuffer.from_flat(gflat))
    mo = AdamMomentBuffers(ctx, n)
    cfg_pos = AdamConfig(lr=k["step_all_pos_lr"])
    cfg_attr = AdamConfig()
    AdamGpu(ctx).step_all(g, grads, mo, 1, cfg_pos, cfg_attr)
    back = g.readback().flat()
    mm, vv = mo.download(n)
    # oracle: six per-attribute Adam slabs (train.rs:84-89)
    flat = s.flat()
    spans = [(0, 3), (3, 7), (7, 10), (10, 11), (11, 14), (14, 59)]
    for j, (a, b) in enumerate(spans):
        lr = cfg_pos.lr if j == 0 else cfg_attr.lr
        p, m, v = oracle.adam_step(flat[:, a:b], gflat[:, a:b], np.zeros((n, b - a)), np.zeros((n, b - a)), lr, 1)
        assert np.abs(back[:, a:b] - p.reshape(n, b - a)).max() < 1e-4
        assert np.allclose(back[:, a:b], p.reshape(n, b - a), rtol=1e-6, atol=1e-7)
        assert np.abs(mm.flat()[:, a:b] - m.reshape(n, -1)).max() < 1e-5
        assert np.abs(vv.flat()[:, a:b] - v.reshape(n, -1)).max() < 1e-5


def test_constraints_and_accumulate_vs_oracle(ctx, oracle):
    s = random_scene(1000, seed=12)
    f = s.flat()
    f[:, 3:7] *= 3.0
    f[:5, 3:7] = 0.0  # zero quaternion: clamped norm 1e-8, no NaN (apply_constraints.wgsl:30-33)
    f[:, 7:10] = np.random.default_rng(1).normal(0, 8, (1000, 3))
    f[:, 10] = np.random.default_rng(2).normal(0, 20, 1000)
    s = SplatBuffer.from_flat(f)
    g = GpuSplatBuffer.upload(ctx, s)
    AdamGpu(ctx).apply_constraints(g)
    back = g.readback()
    rot, sc, op = oracle.apply_constraints(s.rotations, s.scales, s.opacities)
    assert np.allclose(back.rotations, rot.reshape(-1, 4), rtol=1e-6, atol=1e-7)
    assert np.array_equal(back.scales, sc.reshape(-1, 3)) and np.array_equal(back.opacities, op)
    assert np.all(np.isfinite(back.rotations))
    # accumulate_grad_pos
    grads = GradSplatBuffers(ctx, 1000)
    gs = random_scene(1000, seed=13)
    grads.upload(gs)
    acc0 = np.random.default_rng(4).random(1000).astype(np.float32)
    acc = ctx.storage_buffer("acc", acc0)
    AdamGpu(ctx).accumulate_grad(grads, acc, 1000)
    assert np.allclose(acc.readback(np.float32), oracle.accumulate_grad(gs.positions, acc0), rtol=1e-6)


def _gpu_state(ctx, s, m, v, acc, cap):
    g = GpuSplatBuffer.upload(ctx, s, capacity=cap)
    mo = AdamMomentBuffers.upload_from_cpu(ctx, m, v, capacity=cap)
    a = np.zeros(g.capacity, np.float32)
    a[: len(acc)] = acc
    return g, mo, ctx.storage_buffer("acc", a)


def test_densify_kat_on_gpu(ctx):
    k = KATS["densify_clones_small_and_splits_large"]
    sp = k["splats"]
    s = SplatBuffer([x["pos"] for x in sp], [x["rot"] for x in sp], [x["scale"] for x in sp],
                    [x["opacity"] for x in sp], [x["dc"] for x in sp], np.zeros((3, 45)))
    z = SplatBuffer.zeros(3)
    g, mo, acc = _gpu_state(ctx, s, z, z, k["grad_acc"], 16)
    c = densify(ctx, g, mo, acc, k["grad_count"], k["threshold"], k["split_thr"], k["max_splats"], k["iter"])
    ex = k["expect"]
    assert c == (ex["cloned"], ex["split_children"], ex["removed"]) and g.n == ex["len"]


def test_prune_kat_on_gpu(ctx):
    k = KATS["prune_drops_low_opacity_splats"]
    n = len(k["opacities"])
    s = SplatBuffer([[i, i, i] for i in range(n)], [[1, 0, 0, 0]] * n, [[-1, -1, -1]] * n, k["opacities"],
                    np.zeros((n, 3)), np.zeros((n, 45)))
    z = SplatBuffer.zeros(n)
    g, mo, acc = _gpu_state(ctx, s, z, z, k["grad_acc"], n)
    assert prune_low_opacity(ctx, g, mo, acc, k["threshold"]) == k["expect"]["removed"]
    assert g.n == 3 and np.allclose(g.readback().opacities, 2.0)


def _random_state(n, seed):
    rng = np.random.default_rng(seed)
    s = random_scene(n, seed)
    f = s.flat()
    f[:, 10] = np.where(rng.random(n) < 0.3, -8.0, f[:, 10])  # ~30% prunable
    f[:, 7:10] += np.where(rng.random((n, 1)) < 0.4, 3.0, 0.0)  # mix of large and small splats
    s = SplatBuffer.from_flat(f)
    m = SplatBuffer.from_flat(rng.normal(size=(n, 59)).astype(np.float32))
    v = SplatBuffer.from_flat(np.abs(rng.normal(size=(n, 59))).astype(np.float32))
    acc = (rng.random(n) * 4e-4).astype(np.float32)
    return s, m, v, acc


@pytest.mark.parametrize("n,seed", [(1, 0), (97, 1), (5000, 2), (200_003, 3)])
def test_prune_matches_oracle_swap_remove_order(ctx, oracle, n, seed):
    s, m, v, acc = _random_state(n, seed)
    g, mo, accb = _gpu_state(ctx, s, m, v, acc, n)
    removed = prune_low_opacity(ctx, g, mo, accb, -5.3)
    os_, om, ov = oracle.OSplats.from_buffer(s), oracle.OSplats.from_buffer(m), oracle.OSplats.from_buffer(v)
    oacc = acc.copy()
    oremoved = oracle.prune(os_, om, ov, oacc, -5.3)
    assert removed == oremoved and g.n == os_.n
    assert np.array_equal(g.readback().flat(), os_.flat())
    gm, gv = mo.download(g.n)
    assert np.array_equal(gm.flat(), om.flat()) and np.array_equal(gv.flat(), ov.flat())
    assert np.array_equal(accb.readback(np.float32, g.n), oacc[: g.n])


@pytest.mark.parametrize("n,max_splats,it", [(50, 1000, 100), (5000, 6000, 200), (4000, 4000, 400),
                                             (100_000, 180_000, 1000)])
def test_densify_matches_oracle_swap_remove_order(ctx, oracle, n, max_splats, it):
    s, m, v, acc = _random_state(n, it)
    cap = max(max_splats, n)
    g, mo, accb = _gpu_state(ctx, s, m, v, acc, cap)
    c = densify(ctx, g, mo, accb, 1, 2e-4, -2.3, max_splats, it)
    os_ = oracle.OSplats.from_buffer(s, cap)
    om, ov = oracle.OSplats.from_buffer(m, cap), oracle.OSplats.from_buffer(v, cap)
    oacc = np.zeros(n + 2 * max(0, max_splats - n), np.float32)
    oacc[:n] = acc
    oc = oracle.densify(os_, om, ov, oacc, 1, 2e-4, -2.3, max_splats, it)
    assert c == oc and g.n == os_.n
    got, want = g.readback().flat(), os_.flat()
    pos_close = np.abs(got[:, :3] - want[:, :3]) <= 1e-5 * np.maximum(1.0, np.abs(want[:, :3]))
    assert pos_close.all()
    assert np.array_equal(got[:, 3:], want[:, 3:])
    gm, gv = mo.download(g.n)
    assert np.array_equal(gm.flat(), om.flat()) and np.array_equal(gv.flat(), ov.flat())
    assert np.array_equal(accb.readback(np.float32, g.n), oacc[: g.n])


def test_bf16_parameters_round_stochastically_so_small_updates_survive(ctx):
    """With BF16 SH-rest storage, an Adam step smaller than half a BF16 ulp
    would vanish under round-to-nearest.  The parameters are written back with
    stochastic rounding instead: each coefficient moves by one ulp or not at
    all, and over many coefficients the mean change equals the f32 update."""
    n, lr = 4096, 1e-5
    flat = np.zeros((n, 59), np.float32)
    flat[:, 3] = 1.0                  # unit quaternions
    flat[:, 14:] = 0.05               # SH rest: BF16 spacing 2^-12 = 2.4e-4 here
    g = GpuSplatBuffer.upload(ctx, SplatBuffer.from_flat(flat), bf16_rest=True)
    before = g.readback().flat()[:, 14:].astype(np.float64)
    gflat = np.zeros((n, 59), np.float32)
    gflat[:, 14:] = 1.0               # first Adam step: every SH-rest value moves by -lr in f32
    grads = GradSplatBuffers(ctx, n)
    grads.upload(SplatBuffer.from_flat(gflat))
    mo = AdamMomentBuffers(ctx, n)
    AdamGpu(ctx).step_all(g, grads, mo, 1, AdamConfig(lr=lr))
    d = g.readback().flat()[:, 14:].astype(np.float64) - before
    ulp = 2.0 ** -12
    assert np.all((d == 0.0) | (d == -ulp))
    # mean of 184,320 draws with p = lr / ulp: standard error 1.1e-7, bound 5e-7
    assert abs(d.mean() + lr) < 0.05 * lr
