"""Checkpoint and resume (checkpoint.py): host round trip on CPU; the
device round trip and an interrupted-then-resumed run on the GPU."""
import numpy as np
import pytest

from nanotracer_b200.checkpoint import load_checkpoint, save_checkpoint, sidecar
from nanotracer_b200.scene import perturbed, random_scene


def test_host_checkpoint_roundtrip_is_bit_exact(tmp_path):
    s = random_scene(257, 3)
    m, v = perturbed(s, seed=1), perturbed(s, seed=2)
    acc = np.random.default_rng(0).random(257).astype(np.float32)
    p = tmp_path / "ck.ply"
    save_checkpoint(p, s, m, v, 123, acc, 7)
    ck = load_checkpoint(p)
    assert ck.t == 123 and ck.grad_count == 7
    for a, b in ((ck.splats, s), (ck.m, m), (ck.v, v)):
        assert np.array_equal(a.flat(), b.flat())
    assert np.array_equal(ck.grad_acc, acc)


def test_checkpoint_rejects_mismatched_sidecar(tmp_path):
    s = random_scene(10, 3)
    save_checkpoint(tmp_path / "a.ply", s, s, s, 1)
    save_checkpoint(tmp_path / "b.ply", random_scene(11, 3), random_scene(11, 4), random_scene(11, 5), 1)
    sidecar(tmp_path / "b.ply").replace(sidecar(tmp_path / "a.ply"))
    with pytest.raises(ValueError):
        load_checkpoint(tmp_path / "a.ply")
    with pytest.raises(ValueError):
        save_checkpoint(tmp_path / "c.ply", s, random_scene(9, 1), s, 1)


@pytest.mark.gpu
def test_resumed_run_continues_the_uninterrupted_one(ctx, tmp_path):
    from nanotracer_b200.checkpoint import load_device_checkpoint, save_device_checkpoint
    from tests.test_gpu_trainer import _run, _setup
    from nanotracer_b200 import Trainer
    scene, tl, cams, tgt, cfg = _setup(ctx, n=2000, V=2)
    _, g_full, mo_full, acc_full, _ = _run(ctx, scene, cams, tgt, cfg, steps=4)
    # two steps, checkpoint, fresh objects from the checkpoint, two more steps
    tr, g, mo, acc, _ = _run(ctx, scene, cams, tgt, cfg, steps=2)
    save_device_checkpoint(tmp_path / "ck.ply", ctx, g, mo, acc, 2, 2)
    g2, mo2, acc2, t, gc = load_device_checkpoint(tmp_path / "ck.ply", ctx)
    assert t == 2 and gc == 2
    assert np.array_equal(g2.readback().flat(), g.readback().flat())
    tr2 = Trainer(ctx, cfg)
    tb = ctx.storage_buffer("t", np.ascontiguousarray(tgt, np.float32))
    tr2.set_targets(tb)
    for step in (3, 4):
        tr2.step(g2, mo2, acc2, cams, step)
    # the blend's float atomics reorder sums between runs: compare to rounding
    assert np.allclose(g2.readback().flat(), g_full.readback().flat(), rtol=1e-5, atol=1e-7)
    m_a, v_a = mo2.download(len(scene))
    m_b, v_b = mo_full.download(len(scene))
    assert np.allclose(m_a.flat(), m_b.flat(), rtol=1e-4, atol=1e-12)
    assert np.allclose(v_a.flat(), v_b.flat(), rtol=1e-4, atol=1e-18)
