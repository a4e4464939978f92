"""Many scenes in one launch per stage (sc_scenes_trainer): scenes of uneven
splat counts and image sizes stepped together give, scene by scene, the
step of a single-scene trainer on that scene (the same images bit for bit,
the same loss, the same first Adam step up to float summation order), and
agree with the oracle scene by scene; densify and prune run per scene under
a shared total cap."""
import numpy as np
import pytest

from nanotracer_b200 import AdamMomentBuffers, CameraUniform, GpuSplatBuffer, TilingParams, TrainConfig, Trainer
from nanotracer_b200._lib import SC_KEYS_REF32
from nanotracer_b200.scene import FOV_Y, orbit_views, perturbed, random_scene
from nanotracer_b200.scenes import Scene, ScenesTrainer, densify_prune_scenes
from nanotracer_b200.train import BENCH_LRS, render_targets

from tests.util import GpuPipe, check_image_explained, check_same_first_step, margins

pytestmark = pytest.mark.gpu

# (splats, width, height, seed): uneven counts and image sizes inside a 160 x 128 grid
SCENES = [(3000, 160, 128, 31), (12000, 96, 128, 32), (800, 128, 96, 33), (6000, 160, 80, 34)]
MAX_W, MAX_H = 160, 128


def _setup(ctx, specs=SCENES, step=0):
    out = []
    for i, (n, W, H, seed) in enumerate(specs):
        s = random_scene(n, seed)
        cam = CameraUniform.from_pose(*orbit_views(4, step)[i % 4], FOV_Y, W, H, n)
        tgt = render_targets(ctx, perturbed(s), [cam], TilingParams(W, H, 16, 8.0))[0]
        out.append((s, cam, tgt))
    return out


def test_scenes_step_equals_single_scene_trainers(ctx):
    data = _setup(ctx)
    st = ScenesTrainer(ctx, len(SCENES), MAX_W, MAX_H)
    for i, (s, cam, tgt) in enumerate(data):
        st.set_scene(i, Scene.upload(ctx, s, tgt))
    losses = st.step([d[1] for d in data], 1)
    imgs = st.images()
    for i, ((s, cam, tgt), (n, W, H, _)) in enumerate(zip(data, SCENES)):
        g = GpuSplatBuffer.upload(ctx, s)
        mo = AdamMomentBuffers(ctx, g.capacity)
        acc = ctx.storage_buffer_zeroed("acc", 4 * g.capacity)
        tr = Trainer(ctx, TrainConfig(n_views=1, width=W, height=H, depth_max=8.0))
        tr.set_targets(ctx.storage_buffer("t", np.ascontiguousarray(tgt, np.float32)))
        loss = tr.step(g, mo, acc, [cam], 1)
        assert np.array_equal(imgs[i], tr.images()[0]), i
        assert abs(losses[i] - loss) <= 1e-9 * loss, (i, losses[i], loss)
        print(i, check_same_first_step(st.scenes[i].splats.readback().flat(), g.readback().flat(), BENCH_LRS))
        assert np.array_equal(st.scenes[i].grad_acc.readback(np.float32, n) > 0,
                              acc.readback(np.float32, n) > 0)


def test_scenes_match_the_oracle_scene_by_scene(ctx, oracle):
    """Each scene's loss within 1e-5 of the oracle's f32 iteration on that
    scene alone, and its image within 1e-4 of the oracle's blend of the
    scene's records except near-threshold pixels."""
    data = _setup(ctx, step=2)
    st = ScenesTrainer(ctx, len(SCENES), MAX_W, MAX_H)
    for i, (s, cam, tgt) in enumerate(data):
        st.set_scene(i, Scene.upload(ctx, s, tgt))
    losses = st.step([d[1] for d in data], 1)
    imgs = st.images()
    for i, ((s, cam, tgt), (n, W, H, _)) in enumerate(zip(data, SCENES)):
        os_ = oracle.OSplats.from_buffer(s)
        om, ov = oracle.OSplats.zeros(n), oracle.OSplats.zeros(n)
        otl = oracle.tiling(W, H, 16, 16, 8.0)
        ol, _ = oracle.train_step(os_, om, ov, np.zeros(n, np.float32), [oracle.camera_from_struct(bytes(cam.c))],
                                  tgt, otl, 1, BENCH_LRS, 1)
        assert abs(losses[i] - ol) <= 1e-5 * ol, (i, losses[i], ol)
        pipe = GpuPipe(ctx, s, cam, TilingParams(W, H, 16, 8.0), key_mode=SC_KEYS_REF32)
        rec = pipe.project()[0]
        _, pay, ranges = pipe.bin()
        oimg, _, _ = oracle.composite(rec, pay, ranges.reshape(-1), otl)
        m, _, _ = margins(oracle, rec, pay, ranges, otl, 1)
        print(i, check_image_explained(imgs[i], oimg, m, label=f"scene {i}"))


def test_scenes_densify_and_prune_per_scene_under_a_total_cap(ctx):
    """The reference's schedule per scene (prune after 50 every 100, densify
    after 100 every 200), the densify budget shared so the total stays under
    the cap, training continuing with the changed stores (the trainer's grids
    follow the capacities, the counts come with each step)."""
    specs = [(1500, 96, 96, 41), (4000, 128, 96, 42), (700, 64, 64, 43)]
    data = _setup(ctx, specs)
    st = ScenesTrainer(ctx, len(specs), 128, 96)
    caps = [3 * n for n, *_ in specs]
    for i, (s, cam, tgt) in enumerate(data):
        st.set_scene(i, Scene.upload(ctx, s, tgt, capacity=caps[i]))
    cams = [d[1] for d in data]
    max_total = sum(n for n, *_ in specs) + 2000
    counts = []
    for it in range(1, 201):
        losses = st.step(cams, it)
        assert np.all(np.isfinite(losses))
        ev = densify_prune_scenes(st, it, grad_count=100, max_total=max_total,
                                  prune_every=50, prune_warmup=25, densify_every=100, densify_warmup=50)
        counts.append((it, [s.splats.n for s in st.scenes], ev))
    total = sum(s.splats.n for s in st.scenes)
    assert total <= max_total
    assert any(e["pruned"] or e["cloned"] or e["split"] for _, _, e in counts)
    print(counts[-1], [c for c in counts if any(c[2].values())])
